"""The FP64 restatement of the FFA search (oracle/ffa64_oracle.c) against the
bit-exact FP32 one (oracle/gaffa_oracle.c): transform rows and boxcar S/N of
every evaluated row and width agree within the specified tolerance of 1e-5
relative (absolute below |S/N| = 1, where a relative bound means nothing)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from oracle import oracle  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

SNR_RTOL = 1e-5          # relative, |S/N| >= 1
TRANSFORM_RTOL = 1e-5    # of the block's largest magnitude


def snr_close(a, b):
    return np.abs(a - b) <= SNR_RTOL * np.maximum(1.0, np.abs(b))


@pytest.mark.parametrize("rows,bins", [(8, 8), (5, 4), (37, 181), (300, 256), (1023, 200)])
def test_fp64_transform_matches_fp32_transform(rows, bins):
    port = Oracle("port")
    rng = np.random.default_rng(rows * 1000 + bins)
    x = rng.normal(size=rows * bins).astype(np.float32)
    t32 = port.ffa_transform(x, bins).astype(np.float64)
    t64 = oracle.ffa64_transform(x.astype(np.float64), bins)
    scale = np.abs(t64).max()
    assert np.abs(t32 - t64).max() <= TRANSFORM_RTOL * scale


def test_fp64_transform_is_exact_on_the_riptide_golden():
    """8 x 8 identity-like input of the reference's ffa tests: every value is a
    small integer, so FP64 and FP32 agree exactly."""
    port = Oracle("port")
    x = np.zeros((8, 8), np.float32)
    x[np.arange(8), np.arange(8)] = 1.0
    assert np.array_equal(oracle.ffa64_transform(x, 8), port.ffa_transform(x.ravel(), 8).astype(np.float64))


def test_fp32_snr_within_tolerance_of_fp64_for_every_row_and_width():
    """A plain-workload plan (periods 0.2-2 s at 64 us, widths 1..32) on a
    normalised noise series with a weak pulse: each task searched by the
    FP32 oracle with no effective threshold, so every (row, width) yields a
    peak, compared with the FP64 grid of the same task."""
    port = Oracle("port")
    n, tsamp = 1 << 17, 64e-6
    rng = np.random.default_rng(7)
    x = rng.normal(size=n).astype(np.float32)
    ph = (np.arange(n) * tsamp / 0.5) % 1.0
    x += (0.8 * np.exp(-0.5 * ((ph - 0.3) / 0.004) ** 2)).astype(np.float32)
    x = ((x - x.mean()) / x.std()).astype(np.float32)
    tasks, _ = port.make_plan(n, tsamp, 0.2, 2.0)
    widths = np.array([1, 2, 4, 8, 16, 32], np.uint64)
    worst = 0.0
    nrows = 0
    for i in range(0, len(tasks), 7):  # every 7th task: all octaves, small and large rows
        t = tasks[i:i + 1]
        peaks = port.ffa_search(x, t, widths, snr_threshold=-1e30)
        s64, _ = oracle.ffa64_task_snr(x, t[0], widths)
        re = int(t[0]["rows_eval"])
        assert len(peaks) == re * len(widths)
        got = np.zeros((re, len(widths)))
        got[peaks["shift"].astype(int), peaks["width_index"].astype(int)] = peaks["snr"]
        assert snr_close(got, s64).all()
        worst = max(worst, float((np.abs(got - s64) / np.maximum(1.0, np.abs(s64))).max()))
        nrows += re
    assert nrows > 1000
    assert worst < SNR_RTOL
