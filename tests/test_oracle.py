"""Pins the CPU oracle (C restatement) before anything is checked against it.

1. Known-answer vectors from the reference's own C++ tests, restated here
   (file:line of lintian233/gaffa tests/cpp cited on each test).
2. Bit-exact agreement with fixtures produced by the reference's own CPU
   sources (tests/golden/make_golden.py).
"""
import numpy as np
import pytest

from oracle.oracle import OracleError


def flat(rows):
    return np.array(rows, np.float32).reshape(-1)


FFA_IN_8X8 = flat([[0, 0, 0, 0, 0, 0, 0, 1]] * 8)
FFA_OUT_8X8 = flat([
    [0, 0, 0, 0, 0, 0, 0, 8], [0, 0, 0, 0, 0, 0, 4, 4], [0, 0, 0, 0, 0, 2, 4, 2],
    [0, 0, 0, 0, 2, 2, 2, 2], [0, 0, 0, 1, 2, 2, 2, 1], [0, 0, 1, 2, 1, 1, 2, 1],
    [0, 1, 1, 1, 2, 1, 1, 1], [1, 1, 1, 1, 1, 1, 1, 1]])


def test_ffa_riptide_8x8(port):
    # test_ffa.cpp:44-84 MatchesRiptideHandCalculatedEightByEight
    assert np.array_equal(port.ffa_transform(FFA_IN_8X8, 8).reshape(-1), FFA_OUT_8X8)


def test_ffa_odd_rows_golden(port):
    # test_ffa.cpp:86-105 MatchesOddRowGoldenTransform
    x = flat([[1, 2, 3, 4], [5, 6, 7, 8], [9, 10, 11, 12], [13, 14, 15, 16], [17, 18, 19, 20]])
    want = flat([[45, 50, 55, 60], [46, 51, 56, 57], [50, 55, 56, 49], [52, 53, 54, 51],
                 [51, 52, 53, 54]])
    assert np.array_equal(port.ffa_transform(x, 4).reshape(-1), want)


@pytest.mark.parametrize("shift", range(8))
def test_ffa_rotation_invariance(port, shift):
    # test_ffa.cpp:107-120 IsPhaseRotationInvariant
    rot = lambda a: np.roll(a.reshape(8, 8), shift, axis=1).reshape(-1)
    assert np.array_equal(port.ffa_transform(rot(FFA_IN_8X8), 8).reshape(-1), rot(FFA_OUT_8X8))


def test_ffa_ignores_tail_and_zero_columns(port):
    # test_ffa.cpp:122-152 PreservesExtraZeroColumns / IgnoresIncompleteTailSamples
    x = np.concatenate([FFA_IN_8X8, [42.0, 43.0]]).astype(np.float32)
    assert np.array_equal(port.ffa_transform(x, 8).reshape(-1), FFA_OUT_8X8)
    for extra in range(1, 8):
        xin = np.zeros((8, 8 + extra), np.float32)
        xin[:, :8] = FFA_IN_8X8.reshape(8, 8)
        want = np.zeros((8, 8 + extra), np.float32)
        want[:, :8] = FFA_OUT_8X8.reshape(8, 8)
        assert np.array_equal(port.ffa_transform(xin.reshape(-1), 8 + extra), want)


def test_plan_widths_like_riptide(port):
    # test_ffa_plan.cpp:78-91 GeneratesWidthTrialsLikeRiptide
    _, w = port.make_plan(1000, 1.0, 240.0, 300.0, bins_min=240, bins_max=260)
    assert list(w) == [1, 2, 3, 4, 6, 9, 13, 19, 28, 42]


def test_plan_small_known(port):
    # test_ffa_plan.cpp:93-116 MatchesSmallKnownPlan
    t, w = port.make_plan(64, 0.25, 1.0, 4.0, bins_min=4, bins_max=5, min_periods=2,
                          duty_cycle_max=0.5, max_tasks=1000)
    assert len(t) == 7 and list(w) == [1, 2]
    first, last = t[0], t[-1]
    assert first["downsample_factor"] == 1.0 and first["effective_tsamp"] == 0.25
    assert (first["input_nsamples"], first["prepared_nsamples"], first["bins"],
            first["rows"], first["rows_eval"]) == (64, 64, 4, 16, 12)
    assert first["period_begin"] == 1.0
    assert abs(first["period_end"] - 1.2244897959183674) < 1e-12
    assert (last["bins"], last["rows"], last["rows_eval"]) == (4, 4, 2)
    assert last["period_begin"] == 3.375
    assert abs(last["period_end"] - 3.681818181818182) < 1e-12


def test_plan_rejections(port):
    # test_ffa_plan.cpp:40-76, :155-181
    with pytest.raises(OracleError):
        port.make_plan(64, 0.25, 1.0, 4.0, bins_min=4, bins_max=5, min_periods=2,
                       duty_cycle_max=0.5, max_tasks=1)
    with pytest.raises(OracleError):
        port.make_plan(64, 0.25, 4.0, 8.0, bins_min=4, bins_max=5, min_periods=8)
    with pytest.raises(OracleError):
        port.make_plan(64, 0.25, 0.5, 4.0, bins_min=4, bins_max=5)


def test_downsample_known_cases(port):
    # test_time_series.cpp:107-146
    assert np.array_equal(port.downsample([1, 2, 3, 4], 2.0), [3.0, 7.0])
    assert np.array_equal(port.downsample([1, 2, 3, 4, 5], 2.5), np.float32([4.5, 10.5]))
    got = port.downsample([1, 2, 3, 4, 5, 6], 2.25)
    assert np.array_equal(got, np.float32([1 + 2 + 0.25 * 3, 0.75 * 3 + 4 + 0.5 * 5]))


def test_downsampled_variance_known_cases(port):
    # test_time_series.cpp:148-153
    assert abs(port.downsampled_variance(16, 2.0) - 2.0) < 1e-12
    assert abs(port.downsampled_variance(16, 4.0) - 10.0) < 1e-12
    assert abs(port.downsampled_variance(8, 2.5) - (2.5 - 1.0 / 3.0)) < 1e-12
    assert abs(port.downsampled_variance(5, 2.5) - 5.0 / 3.0) < 1e-12


def _detrend(port, x, window, min_points):
    import ctypes as C
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    f = port.lib.gfo_detrend_running_median
    rc = f(x.ctypes.data_as(C.POINTER(C.c_float)), C.c_uint64(len(x)), C.c_uint64(window),
           C.c_uint64(min_points), out.ctypes.data_as(C.POINTER(C.c_float)))
    assert rc == 0
    return out


def test_detrend_known_cases(port):
    # test_preprocessing.cpp:114-127 ExactRunningMedianUsesRiptideEdgePadding
    assert np.array_equal(_detrend(port, [100, 0, 1, 2, 3], 3, 101), [0, -1, 0, 0, 0])
    # test_preprocessing.cpp:129-149 FastRunningMedianScrunchesAndInterpolates
    out = _detrend(port, [1, 1, 1, 9, 9, 9, 1, 1, 1, 9, 9, 9], 7, 3)
    assert [out[i] for i in (0, 1, 2, 3, 9, 10, 11)] == [0, -1, -3, 4, 3, 1, 0]
    # test_preprocessing.cpp:151-162 RunningMedianDetrendPreservesLengthAndRemovesBaseline
    assert np.array_equal(_detrend(port, [10, 10, 20, 10, 10], 3, 101), [0, 0, 10, 0, 0])


def test_subband_dm_zero_sums(port):
    # test_dedispersion.cpp:298-314 SubbandNormalModeProducesExpectedDmZeroSums
    data = np.array([[1, 2, 3, 4], [5, 6, 7, 8]], np.uint8)
    out = port.dedisperse_subband(data, [1000.0, 1200.0, 1500.0, 2000.0], 0.0, 1.0, 1,
                                  2000.0, 1.0, 2, 32)
    assert out.tolist() == [[10, 26]]


@pytest.mark.parametrize("sbc", [1, 3, 8])
def test_degenerate_subband_equals_multi_dm(port, sbc):
    # test_dedispersion.cpp:435-497: with one DM per nominal DM the stage-2
    # residual delays vanish, so the subband sums equal the direct sums
    rng = np.random.default_rng(sbc)
    data = rng.integers(0, 256, (3000, 24), dtype=np.uint8)
    freq = np.linspace(1500.0, 1200.0, 24)
    multi = port.dedisperse_multi_dm(data, freq, 2.0, 3.5, 17, 1500.0, 1e-3)
    sub = port.dedisperse_subband(data, freq, 2.0, 3.5, 17, 1500.0, 1e-3, sbc, 1)
    assert sub.shape == multi.shape and np.array_equal(sub, multi)
    from oracle.oracle import Oracle
    if Oracle.available("reference"):
        # and the reference's own subband code agrees with the restatement,
        # degenerate or not
        ref = Oracle("reference")
        for npn in (1, 4):
            assert np.array_equal(ref.dedisperse_subband(data, freq, 2.0, 3.5, 17, 1500.0, 1e-3, sbc, npn),
                                  port.dedisperse_subband(data, freq, 2.0, 3.5, 17, 1500.0, 1e-3, sbc, npn))


def test_single_dm_is_a_prefix_of_the_multi_dm_row(port):
    # test_dedispersion.cpp:435-497: one DM's own series (its aligned spectrum
    # summed over channels, valid over its own delay) starts with that DM's
    # row of the multi-DM block (valid over the highest DM's delay)
    rng = np.random.default_rng(7)
    data = rng.integers(0, 256, (4000, 32), dtype=np.uint8)
    freq = np.linspace(1500.0, 1200.0, 32)
    multi = port.dedisperse_multi_dm(data, freq, 0.0, 4.0, 12, 1500.0, 1e-3)
    for i in (0, 5, 11):
        single = port.dedisperse_spectrum(data, freq, 4.0 * i, 1500.0, 1e-3).astype(np.uint32).sum(axis=1)
        assert len(single) >= multi.shape[1]
        assert np.array_equal(single[: multi.shape[1]], multi[i])


def _riptide_snr(bins, width, boxsum, total, stdnoise):
    # test_ffa_detection.cpp:24-33 expected_riptide_snr (float arithmetic)
    b, w = np.float32(bins), np.float32(width)
    h = np.sqrt((b - w) / (b * w), dtype=np.float32)
    beta = w / (b - w) * h
    return np.float32(((h + beta) * np.float32(boxsum) - beta * np.float32(total))
                      * (np.float32(1.0) / np.float32(stdnoise)))


def _task(rows, bins, tsamp=0.25):
    from oracle.oracle import TASK_DTYPE
    t = np.zeros(1, TASK_DTYPE)
    t["downsample_factor"] = 1.0
    t["effective_tsamp"] = tsamp
    t["input_nsamples"] = rows * bins
    t["prepared_nsamples"] = rows * bins
    t["bins"], t["rows"], t["rows_eval"] = bins, rows, rows
    return t


def _find(port, transform, rows, bins, widths, task=None):
    import ctypes as C
    from oracle.oracle import PEAK_DTYPE
    task = _task(rows, bins) if task is None else task
    tr = np.ascontiguousarray(transform, np.float32)
    w = np.ascontiguousarray(widths, np.uint64)
    pp, n = C.c_void_p(), C.c_uint64()
    rc = port.lib.gfo_find_ffa_peaks(
        tr.ctypes.data_as(C.POINTER(C.c_float)), C.c_uint64(rows), C.c_uint64(bins),
        task.ctypes.data_as(C.c_void_p), w.ctypes.data_as(C.POINTER(C.c_uint64)),
        C.c_uint64(len(w)), C.c_float(1.0), C.c_float(0.0), C.c_uint64(0),
        C.byref(pp), C.byref(n))
    assert rc == 0
    return port._take(pp, n.value, PEAK_DTYPE)


def test_detection_known_cases(port):
    # test_ffa_detection.cpp:155-176 DetectsSingleBinPeak
    p = _find(port, [0, 0, 5, 0], 1, 4, [1])
    assert len(p) == 1 and p[0]["phase"] == 2 and p[0]["period"] == 1.0
    assert p[0]["duty_cycle"] == 0.25 and p[0]["snr"] == _riptide_snr(4, 1, 5, 5, 1)
    # :178-191 DetectsCircularBoxcarAcrossBoundary
    p = _find(port, [4, 0, 0, 5], 1, 4, [2])
    assert p[0]["phase"] == 3 and p[0]["snr"] == _riptide_snr(4, 2, 9, 9, 1)
    # :193-207 KeepsFirstPhaseWhenBoxcarSumsTie
    p = _find(port, [1, 1, 0, 1, 1, 0], 1, 6, [2])
    assert p[0]["phase"] == 0 and p[0]["snr"] == _riptide_snr(6, 2, 2, 4, 1)
    # :209-231 ComputesPeriodFromTaskRowsNotRowsEval
    t = _task(4, 4)
    t["rows"] = 8
    tr = np.zeros(16, np.float32)
    tr[3 * 4 + 1] = 10.0
    p = _find(port, tr, 4, 4, [1], task=t)
    sel = p[p["shift"] == 3]
    assert sel[0]["period"] == 0.25 * 4.0 * 4.0 / (4.0 - 3.0 / 7.0)
    # :233-248 SortsPeaksBySnrDescending
    p = _find(port, [0, 0, 2, 0, 0, 0, 8, 0], 2, 4, [1])
    assert p[0]["snr"] > p[1]["snr"] and p[0]["shift"] == 1


SMALL_KEYS_DD = ["dd_multi", "dd_multi_sub", "dd_subband", "dd_subband_ragged"]


def test_port_matches_reference_dedispersion(port, golden_small):
    g = golden_small
    d, f = g["dd_data"], g["dd_freq"]
    assert np.array_equal(port.dedisperse_multi_dm(d, f, 0.0, 2.5, 24, f.max(), 1e-3), g["dd_multi"])
    assert np.array_equal(port.dedisperse_multi_dm(d, f, 3.0, 1.25, 17, f.max(), 1e-3, 5, 61),
                          g["dd_multi_sub"])
    assert np.array_equal(port.dedisperse_subband(d, f, 0.0, 2.5, 24, f.max(), 1e-3, 16, 4),
                          g["dd_subband"])
    assert np.array_equal(port.dedisperse_subband(d, f, 1.0, 1.5, 23, f.max(), 1e-3, 12, 5, 3, 64),
                          g["dd_subband_ragged"])
    from gaffa_b200 import synth
    lv = synth.unpack_2bit(g["dd2_packed"], 64)
    f2 = g["dd2_freq"]
    assert np.array_equal(port.dedisperse_multi_dm(lv, f2, 0.0, 0.5, 20, f2.max(), 1e-3), g["dd2_multi"])
    assert np.array_equal(port.dedisperse_subband(lv, f2, 0.0, 0.5, 20, f2.max(), 1e-3, 16, 8),
                          g["dd2_subband"])


def test_port_matches_reference_preprocess_and_ffa(port, golden_small):
    g = golden_small
    x = g["pp_in"]
    assert np.array_equal(port.preprocess(x, 1e-3, 1.0, 101), g["pp_scrunched"])
    assert np.array_equal(port.preprocess(x, 1e-3, 0.051, 101), g["pp_exact"])
    assert np.array_equal(port.preprocess(x, 1e-3, 1.0, 101, normalise=False), g["pp_scrunched_raw"])
    for name in ("ds_a", "ds_b", "ds_c", "ds_d"):
        fct = float(g[name + "_factor"])
        assert np.array_equal(port.downsample(g["ds_in"], fct), g[name])
        assert port.downsampled_variance(len(g["ds_in"]), fct) == float(g[name + "_var"])
    for key in g:
        if key.startswith("ffa_in_"):
            shape = key[len("ffa_in_"):]
            bins = int(shape.split("x")[1])
            assert np.array_equal(port.ffa_transform(g[key], bins), g["ffa_out_" + shape]), shape
    for key, (n, ts, pmin, pmax, kw) in {
        "plan_a": (29527, 64e-6, 0.2, 2.0, {}),
        "plan_b": (258903, 64e-6, 0.2, 2.0, {}),
        "plan_c": (8357464, 64e-6, 0.1, 10.0, {"duty_cycle_max": 0.1}),
        "plan_d": (64, 0.25, 1.0, 4.0, dict(bins_min=4, bins_max=5, min_periods=2,
                                            duty_cycle_max=0.5, max_tasks=1000)),
    }.items():
        tasks, widths = port.make_plan(n, ts, pmin, pmax, **kw)
        assert np.array_equal(tasks, g[key + "_tasks"]) and np.array_equal(widths, g[key + "_widths"])


def test_port_matches_reference_search_candidates_fold(port, golden_small):
    g = golden_small
    assert np.array_equal(port.ffa_search(g["search_in"], g["search_tasks"], g["search_widths"], 3.0),
                          g["search_peaks"])
    assert np.array_equal(port.ffa_search(g["search_in"], g["search_tasks"],
                                          np.array([1, 2, 5, 11], np.uint64), 2.0),
                          g["search_peaks_w"])
    peaks = port.find_dm_peaks(g["dd_multi"], np.arange(24) * 2.5, 1e-3,
                               dict(period_min=0.1, period_max=1.0, bins_min=40, bins_max=64),
                               dict(window_seconds=0.5, min_points=11), 5.0)
    assert np.array_equal(peaks, g["dm_peaks"])
    tobs = g["dd_multi"].shape[1] * 1e-3
    assert np.array_equal(port.select_candidates(peaks, tobs), g["cands_default"])
    assert np.array_equal(port.select_candidates(peaks, tobs, 0.5, 3, False, 5), g["cands_r3_w"])
    prof, expo = port.fold(g["fold_in_u32"], 0.25, 1e-3, 32)
    assert np.array_equal(prof, g["fold_u32_profile"]) and np.array_equal(expo, g["fold_u32_exposure"])
    prof, expo = port.fold(g["pp_scrunched"], 0.1234, 1e-3, 50, 17)
    np.testing.assert_allclose(prof, g["fold_f32_profile"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(expo, g["fold_f32_exposure"], rtol=1e-12)


def test_port_matches_reference_plain_end_to_end(port, golden_plain):
    """Full 256 ch x 2^18 x 512 DM workload: bit-exact dedispersion digest, the
    exact raw-peak digest and an identical candidate list."""
    import hashlib
    from gaffa_b200 import configs, synth
    g = golden_plain
    cfg = configs.plain_end_to_end()
    obs = cfg.obs
    data = synth.generate(obs)
    assert hashlib.sha256(data.tobytes()).hexdigest() == str(g["input_digest"])
    dd = port.dedisperse_multi_dm(data, obs.frequencies, cfg.dm_low, cfg.dm_step, cfg.ndm,
                                  obs.ref_frequency, obs.tsamp)
    assert hashlib.sha256(dd.tobytes()).hexdigest() == str(g["dedispersed_digest"])
    peaks = port.find_dm_peaks(dd, cfg.dms, obs.tsamp, cfg.plan_options(),
                               cfg.preprocess_options(), cfg.snr_threshold,
                               widths=np.array(cfg.width_trials, np.uint64))
    assert len(peaks) == int(g["npeaks"])
    assert hashlib.sha256(peaks.tobytes()).hexdigest() == str(g["peaks_digest"])
    cands = port.select_candidates(peaks, obs.nsamples * obs.tsamp)
    assert np.array_equal(cands, g["candidates"])
