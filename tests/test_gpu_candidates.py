"""Candidate selection on the device (gf_select_candidates_device) against
the host selection, which restates select_candidates_cpu
(candidate.cpp:175-212) and is pinned to the reference's own candidate lists.

* The plain end-to-end workload (256 channels x 2^18 samples x 512 DMs,
  21.9 million raw peaks) through DmSearch with device_candidates gives the
  reference's 39 candidates and harmonic relations exactly
  (tests/golden/ref_plain_end_to_end.npz, ref_harmonic.npz).
* Randomised FFA searches with low thresholds (10^5-10^6 raw peaks from
  several DM batches), under every candidate option (frequency and DM
  radii, clustering across widths or not, a candidate cap), equal the host
  selection of the same peaks field for field.
"""
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_plain_end_to_end_device_candidates_match_reference(golden_plain):
    from gaffa_b200 import configs, search
    g = golden_plain
    cfg = configs.plain_end_to_end()
    from gaffa_b200 import synth
    data = synth.generate(cfg.obs)
    ds = search.from_config(cfg, dm_batch=128, device_candidates=True)
    res = ds.run(data)
    assert res.peak_count == int(g["npeaks"]) and len(res.peaks) == 0
    assert np.array_equal(res.candidates, g["candidates"])
    h = np.load(Path(__file__).resolve().parent / "golden" / "ref_harmonic.npz")
    assert np.array_equal(res.ranked, h["plain_sorted"])
    assert np.array_equal(res.harmonics, h["plain_rel"])


@pytest.mark.parametrize("seed", [0, 1])
def test_device_selection_equals_host_selection_under_every_option(seed):
    from gaffa_b200 import core
    rng = np.random.default_rng(100 + seed)
    n, tsamp, nser = 40_000, 1e-3, 24
    x = rng.normal(size=(nser, n)).astype(np.float32)
    x[:, ::377] += 1.5                                  # a shared pulse train: clusters across DMs
    plan = core.make_riptide_ffa_plan(n, tsamp, 0.1, 2.0, bins_min=40, bins_max=64)
    prog = core.FfaProgram(plan, max_series=8)
    xs = torch.from_numpy(x).cuda()
    records, segments, hostpeaks, at = [], [], [], 0
    for b0 in range(0, nser, 8):                      # three DM batches
        prep = prog.prepare(xs[b0:b0 + 8], 8)
        rec = prog.search(prep, 8, 3.0)
        records.append(torch.from_numpy(rec.view(np.uint8).copy()).cuda())
        segments.append((at, len(rec), b0))
        at += len(rec)
        hostpeaks.append(prog.expand(rec, b0, 5.0, 0.25))
    peaks = core.sort_peaks(np.concatenate(hostpeaks))
    allrec = torch.cat(records)
    assert len(peaks) > 50_000
    tobs = n * tsamp
    for radius, dm_radius, across, cap in [(0.1, 1, True, 0), (0.5, 3, True, 0), (0.1, 1, False, 0),
                                           (2.0, 0, False, 25), (0.0, 1, True, 0)]:
        want = core.select_candidates(peaks, tobs, radius, dm_radius, across, cap)
        got = core.select_candidates_device(prog, allrec, segments, 5.0, 0.25, tobs, radius, dm_radius, across, cap)
        assert len(got) == len(want) > 0, (radius, dm_radius, across, cap)
        assert np.array_equal(got, want), (radius, dm_radius, across, cap)


def _synthetic_candidates(n, seed):
    """n candidates over 0.1-10 Hz with planted harmonic families (n/m
    multiples of fundamentals within a fraction of a Fourier bin, nearby DMs)
    and noise candidates, ties in S/N and peak counts included."""
    from gaffa_b200 import _lib
    rng = np.random.default_rng(seed)
    tobs = 300.0
    c = np.zeros(n, _lib.CAND_DTYPE)
    nf = n // 8
    f0 = rng.uniform(0.1, 1.0, nf)
    freq = np.empty(n)
    freq[:nf] = f0
    k = np.arange(nf, n)
    num = rng.integers(1, 17, len(k))
    den = rng.integers(1, 6, len(k))
    base = f0[rng.integers(0, nf, len(k))]
    harm = rng.random(len(k)) < 0.6
    freq[nf:] = np.where(harm, base * num / den + rng.normal(0, 0.3 / tobs, len(k)), rng.uniform(0.1, 10.0, len(k)))
    freq = np.abs(freq) + 1e-3
    c["frequency"] = freq
    c["period"] = 1.0 / freq
    c["duty_cycle"] = rng.uniform(0.01, 0.1, n)
    c["dm_index"] = rng.integers(0, 2048, n)
    c["dm"] = c["dm_index"] * 0.4885
    c["snr"] = np.round(rng.uniform(8, 30, n), 1).astype(np.float32)        # many S/N ties
    c["peak_count"] = rng.integers(1, 50, n)
    c["width"] = 4
    return c, tobs


@pytest.mark.parametrize("n,seed", [(39, 0), (3000, 1), (20000, 2)])
def test_device_harmonic_flagging_equals_host(n, seed):
    from gaffa_b200 import core
    if n == 39:
        g = np.load(Path(__file__).resolve().parent / "golden" / "ref_plain_end_to_end.npz")
        cands, tobs = g["candidates"], 2 ** 18 * 64e-6
        lo, hi = 1200.0, 1500.0
    else:
        cands, tobs = _synthetic_candidates(n, seed)
        lo, hi = 1100.0, 1700.0
    host = core.flag_harmonics(cands, tobs, lo, hi, device_id=None) if n < core.DEVICE_HARMONIC_MIN else None
    if host is None:
        from gaffa_b200 import _lib
        import ctypes as C
        ctx = _lib.HarmonicContext(tobs, lo, hi)
        opts = core.harmonic_options()
        out = np.zeros(n, _lib.CAND_DTYPE)
        rel = np.zeros(n, _lib.HARMONIC_DTYPE)
        _lib.check(_lib.lib().gf_flag_harmonics(_lib.ptr(np.ascontiguousarray(cands)), n, C.byref(ctx),
                                                C.byref(opts), _lib.ptr(out), _lib.ptr(rel)))
        host = (out, rel)
    dev = core.flag_harmonics(cands, tobs, lo, hi, device_id=0)
    assert np.array_equal(dev[0], host[0])
    assert np.array_equal(dev[1], host[1])
    if n > 39:
        assert dev[1]["is_harmonic"].sum() > n // 10      # the planted families are found
