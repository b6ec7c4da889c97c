"""Harmonic flagging and removal (src/gaffa/harmonic.cpp) through the C ABI.

Known-answer cases restate tests/cpp/test_harmonic.cpp of the reference;
the seeded candidate lists in tests/golden/ref_harmonic.npz were produced by
the reference's own flag_harmonics_cpu / remove_harmonics_cpu
(tests/golden/make_golden.py).  Host code only: no GPU needed.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from gaffa_b200 import _lib, core

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_harmonic.npz"
CTX = (100.0, 1000.0, 1500.0)  # test_harmonic.cpp:61-66


def cand(dm, dm_index, frequency, snr):
    """test_harmonic.cpp:36-59: width 2, duty 0.02, one peak."""
    c = np.zeros(1, _lib.CAND_DTYPE)[0]
    c["dm"], c["dm_index"], c["period"], c["frequency"] = dm, dm_index, 1.0 / frequency, frequency
    c["width"], c["duty_cycle"], c["snr"], c["peak_count"] = 2, 0.02, snr, 1
    c["dm_index_min"] = c["dm_index_max"] = dm_index
    c["frequency_min"] = c["frequency_max"] = frequency
    bp = c["best_peak"]
    bp["dm"], bp["dm_index"], bp["period"], bp["frequency"] = dm, dm_index, 1.0 / frequency, frequency
    bp["width"], bp["duty_cycle"], bp["width_index"], bp["bins"], bp["snr"] = 2, 0.02, 1, 100, snr
    return c


def cands(*rows):
    return np.array([cand(*r) for r in rows], _lib.CAND_DTYPE)


def flag(c, **opts):
    return core.flag_harmonics(c, *CTX, options=core.harmonic_options(**opts) if opts else None)


def test_empty_input():
    srt, rel = flag(np.zeros(0, _lib.CAND_DTYPE))
    assert len(srt) == 0 and len(rel) == 0


def test_rejects_invalid_inputs():
    c = cands((10.0, 0, 1.0, 5.0))
    with pytest.raises(ValueError, match="observation_seconds"):
        core.flag_harmonics(c, 0.0, 1000.0, 1500.0)
    with pytest.raises(ValueError, match="max_harmonic"):
        flag(c, max_harmonic=1)
    bad = c.copy()
    bad[0]["frequency"] = np.inf
    with pytest.raises(ValueError, match="finite"):
        flag(bad)


def test_integer_harmonic_from_stronger_candidate():
    srt, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, 2.0, 20.0)))
    assert not rel[0]["is_harmonic"]
    assert rel[1]["is_harmonic"] and rel[1]["parent_index"] == 0
    assert (rel[1]["numerator"], rel[1]["denominator"]) == (2, 1)
    assert rel[1]["frequency_error_bins"] == 0.0
    assert rel[0]["parent_index"] == _lib.NO_HARMONIC_PARENT


def test_fractional_harmonic():
    _, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, 1.5, 20.0)), max_harmonic=16, denominator_max=4)
    assert rel[1]["is_harmonic"] and (rel[1]["numerator"], rel[1]["denominator"]) == (3, 2)


def test_default_options_ignore_high_denominator():
    _, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, 10.0 / 9.0, 20.0)))
    assert not rel[1]["is_harmonic"]


@pytest.mark.parametrize("f", [2.02, 2.01])
def test_keeps_candidate_outside_frequency_or_phase_tolerance(f):
    _, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, f, 20.0)))
    assert not rel[1]["is_harmonic"]


def test_keeps_candidate_outside_dm_distance():
    _, rel = flag(cands((10.0, 0, 1.0, 30.0), (1000010.0, 100, 2.0, 20.0)))
    assert not rel[1]["is_harmonic"]


def test_flagged_candidate_is_not_a_parent():
    _, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, 1.5, 20.0), (10.0, 0, 2.25, 10.0)),
                  max_harmonic=3, denominator_max=2)
    assert rel[1]["is_harmonic"] and not rel[2]["is_harmonic"]


def test_snr_consistency_diagnostic_and_hard():
    c = cands((10.0, 0, 1.0, 30.0), (10.0, 0, 2.0, 1.0))
    _, rel = flag(c)
    assert rel[1]["is_harmonic"] and rel[1]["snr_distance"] > 3.0
    assert math.isclose(rel[1]["expected_snr"], 30.0 / math.sqrt(2.0))
    _, rel = flag(c, max_harmonic=16, denominator_max=16, use_snr_consistency=True, snr_distance_max=3.0)
    assert not rel[1]["is_harmonic"]


def test_remove_harmonics_applies_cap():
    srt, rel = flag(cands((10.0, 0, 1.0, 30.0), (10.0, 0, 2.0, 20.0), (10.0, 0, 1.7, 15.0)))
    kept = core.remove_harmonics(srt, rel, 1)
    assert len(kept) == 1 and kept[0]["frequency"] == 1.0
    assert len(core.remove_harmonics(srt, rel)) == 2


def test_ranking_order():
    c = cands((10.0, 3, 1.0, 20.0), (10.0, 1, 3.3, 20.0), (10.0, 2, 1.7, 25.0))
    c[0]["peak_count"] = 5
    srt, _ = flag(c)
    # S/N desc, then peak_count desc
    assert list(srt["dm_index"]) == [2, 3, 1]


def _options(k):
    return [dict(), dict(max_harmonic=8, denominator_max=3),
            dict(frequency_tolerance_bins=3.0, phase_distance_max=2.0, dm_distance_max=10.0),
            dict(use_snr_consistency=True, snr_distance_max=5.0)][k]


@pytest.mark.parametrize("k", range(4))
def test_matches_reference_fixtures(k):
    g = np.load(GOLDEN)
    ctx = tuple(g[f"h{k}_ctx"])
    srt, rel = core.flag_harmonics(g[f"h{k}_in"], *ctx, options=core.harmonic_options(**_options(k)))
    assert np.array_equal(srt, g[f"h{k}_sorted"])
    assert np.array_equal(rel, g[f"h{k}_rel"].astype(_lib.HARMONIC_DTYPE))
    assert np.array_equal(core.remove_harmonics(srt, rel, 10), g[f"h{k}_kept"])


@pytest.mark.parametrize("k", range(4))
def test_oracle_port_matches_reference_fixtures(port, k):
    g = np.load(GOLDEN)
    srt, rel = port.flag_harmonics(g[f"h{k}_in"], *tuple(g[f"h{k}_ctx"]), **_options(k))
    assert np.array_equal(srt, g[f"h{k}_sorted"])
    assert np.array_equal(rel, g[f"h{k}_rel"])
    assert np.array_equal(port.remove_harmonics(srt, rel, 10), g[f"h{k}_kept"])


def test_plain_end_to_end_candidates_match_reference(golden_plain):
    """The 39 candidates of the plain end-to-end workload, flagged with the
    pipeline's context (T = nsamples * tsamp, band 1200-1500 MHz)."""
    g = np.load(GOLDEN)
    srt, rel = core.flag_harmonics(golden_plain["candidates"], *tuple(g["plain_ctx"]))
    assert np.array_equal(srt, g["plain_sorted"])
    assert np.array_equal(rel, g["plain_rel"].astype(_lib.HARMONIC_DTYPE))
    assert rel["is_harmonic"].sum() == 10
