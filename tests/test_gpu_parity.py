"""CUDA path vs the reference: parity through the C ABI on a B200.

Dedispersion, FFA transform rows, prefix sums and S/N values are compared bit
for bit (the kernels keep the reference's operation order); folding, whose
FP64 accumulation order differs like the reference's own OpenMP reduction,
is compared to 1e-6 relative.  Fixtures come from the reference's CPU sources
(tests/golden/make_golden.py); randomised cases use the C restatement.
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FOLD_RTOL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def core():
    from gaffa_b200 import core as c
    return c


def u32(t):
    return t.cpu().numpy().view(np.uint32)


def dedisperse(data, freq, dm_low, dm_step, ndm, tsamp, nbits=8, algorithm="brute", sbc=32, npn=32,
               chan_begin=0, chan_end=None, batch=None):
    c = core()
    prog = c.DedispersionProgram(freq, data.shape[0], tsamp, dm_low, dm_step, ndm, chan_begin=chan_begin,
                                 chan_end=chan_end, nbits=nbits, algorithm=algorithm, subband_channels=sbc,
                                 ndm_per_nominal=npn)
    staged = prog.stage(torch.from_numpy(np.ascontiguousarray(data)).cuda())
    g = prog.batch_granularity
    batch = batch or ndm
    rows = []
    for b0 in range(0, ndm, batch):
        cnt = min(batch, ndm - b0)
        out = prog.run(staged, b0, cnt)
        rows.append(u32(out)[:, : prog.nout])
    return np.concatenate(rows), prog


def test_dedisperse_multi_dm_matches_reference(golden_small):
    g = golden_small
    d, f = g["dd_data"], g["dd_freq"]
    got, _ = dedisperse(d, f, 0.0, 2.5, 24, 1e-3)
    assert np.array_equal(got, g["dd_multi"])
    got, _ = dedisperse(d, f, 3.0, 1.25, 17, 1e-3, chan_begin=5, chan_end=61)
    assert np.array_equal(got, g["dd_multi_sub"])
    got, _ = dedisperse(d, f, 0.0, 2.5, 24, 1e-3, batch=8)  # DM batches
    assert np.array_equal(got, g["dd_multi"])


def test_dedisperse_2bit_matches_reference(golden_small):
    g = golden_small
    got, _ = dedisperse(g["dd2_packed"], g["dd2_freq"], 0.0, 0.5, 20, 1e-3, nbits=2)
    assert np.array_equal(got, g["dd2_multi"])


def test_dedisperse_subband_matches_reference(golden_small):
    g = golden_small
    d, f = g["dd_data"], g["dd_freq"]
    got, _ = dedisperse(d, f, 0.0, 2.5, 24, 1e-3, algorithm="subband", sbc=16, npn=4)
    assert np.array_equal(got, g["dd_subband"])
    got, _ = dedisperse(d, f, 1.0, 1.5, 23, 1e-3, algorithm="subband", sbc=12, npn=5, chan_begin=3)
    assert np.array_equal(got, g["dd_subband_ragged"])
    got, _ = dedisperse(d, f, 0.0, 2.5, 24, 1e-3, algorithm="subband", sbc=16, npn=4, batch=8)
    assert np.array_equal(got, g["dd_subband"])
    got, _ = dedisperse(g["dd2_packed"], g["dd2_freq"], 0.0, 0.5, 20, 1e-3, nbits=2, algorithm="subband",
                        sbc=16, npn=8)
    assert np.array_equal(got, g["dd2_subband"])


@pytest.mark.parametrize("seed", range(6))
def test_dedisperse_random_shapes_match_oracle(port, seed):
    """Ragged channel counts, DM counts that are not multiples of the block and
    tiny time axes, against the C restatement."""
    from gaffa_b200 import synth
    rng = np.random.default_rng(seed)
    nchans = int(rng.choice([1, 3, 17, 64, 100, 257, 300]))
    nsamples = int(rng.integers(1500, 9000))
    obs = synth.Observation(nchans=nchans, nsamples=nsamples, tsamp=1e-3, f_low=1100.0, f_high=1500.0,
                            seed=seed, pulsars=[synth.Pulsar(0.2, 10.0, 0.05, 30.0)])
    data = synth.generate(obs)
    f = obs.frequencies
    ndm = int(rng.integers(1, 40))
    step = float(rng.uniform(0.1, 3.0))
    want = port.dedisperse_multi_dm(data, f, 0.5, step, ndm, f.max(), 1e-3)
    got, _ = dedisperse(data, f, 0.5, step, ndm, 1e-3)
    assert np.array_equal(got, want)


def test_dedisperse_high_channel_count_flushes():
    """More than 256 channels exercises the 16-bit lane flush; compare with the
    oracle on 1100 channels of saturated samples (worst case for the lanes)."""
    from oracle.oracle import Oracle
    port = Oracle("port")
    rng = np.random.default_rng(3)
    data = np.full((3000, 1100), 255, np.uint8)
    data[rng.integers(0, 3000, 500), rng.integers(0, 1100, 500)] = 7
    f = np.linspace(1100.0, 1500.0, 1100)
    want = port.dedisperse_multi_dm(data, f, 0.0, 0.3, 13, f.max(), 1e-3)
    got, _ = dedisperse(data, f, 0.0, 0.3, 13, 1e-3)
    assert np.array_equal(got, want)


def _pre(x, tsamp, window, min_points, normalise=True):
    c = core()
    prog = c.PreprocessProgram(len(x), tsamp, window_seconds=window, min_points=min_points,
                               normalise=normalise, max_series=1)
    t = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda().view(1, -1).clone()
    prog.run(t, 1)
    if normalise:
        prog.normalise_inplace(t, 1)
    prog.synchronize()
    return t.cpu().numpy()[0]


def test_preprocess_matches_reference(golden_small):
    g = golden_small
    x = g["pp_in"]
    assert np.array_equal(_pre(x, 1e-3, 1.0, 101), g["pp_scrunched"])
    assert np.array_equal(_pre(x, 1e-3, 0.051, 101), g["pp_exact"])
    assert np.array_equal(_pre(x, 1e-3, 1.0, 101, normalise=False), g["pp_scrunched_raw"])


def test_preprocess_u32_batch_matches_oracle(port, golden_small):
    c = core()
    blk = golden_small["dd_multi"]
    prog = c.PreprocessProgram(blk.shape[1], 1e-3, window_seconds=0.5, min_points=11, max_series=24)
    t = torch.from_numpy(blk.view(np.int32).copy()).cuda()
    prog.run(t, 24)
    prog.normalise_inplace(t.view(torch.float32), 24)
    prog.synchronize()
    got = t.view(torch.float32).cpu().numpy()
    for i in range(24):
        want = port.preprocess(blk[i].astype(np.float32), 1e-3, 0.5, 11)
        assert np.array_equal(got[i], want), i


def test_preprocess_deferred_errors():
    c = core()
    prog = c.PreprocessProgram(5000, 1e-3, window_seconds=0.5, min_points=11, max_series=2)
    x = torch.ones((2, 5000), dtype=torch.float32, device="cuda")
    prog.run(x, 2)
    with pytest.raises(ValueError, match="standard deviation"):
        prog.synchronize()
    x = torch.randn((2, 5000), device="cuda")
    x[1, 77] = float("nan")
    prog.run(x, 2)
    with pytest.raises(ValueError, match="finite"):
        prog.synchronize()


def test_ffa_transform_matches_reference(golden_small):
    c = core()
    g = golden_small
    for key in g:
        if not key.startswith("ffa_in_"):
            continue
        shape = key[len("ffa_in_"):]
        bins = int(shape.split("x")[1])
        got = c.ffa_transform(torch.from_numpy(g[key]).cuda(), bins).cpu().numpy()
        assert np.array_equal(got, g["ffa_out_" + shape]), shape


def _search(series, tasks, widths, thr):
    c = core()
    plan = c.FfaPlan(tasks, widths)
    prog = c.FfaProgram(plan, max_series=1)
    s = torch.from_numpy(np.ascontiguousarray(series, np.float32)).cuda().view(1, -1)
    prep = prog.prepare(s, 1)
    rec = prog.search(prep, 1, thr)
    return c.sort_peaks(prog.expand(rec))


def test_ffa_search_matches_reference(golden_small):
    g = golden_small
    got = _search(g["search_in"], g["search_tasks"], g["search_widths"], 3.0)
    assert len(got) == len(g["search_peaks"])
    assert np.array_equal(got, g["search_peaks"])
    got = _search(g["search_in"], g["search_tasks"], [1, 2, 5, 11], 2.0)
    assert np.array_equal(got, g["search_peaks_w"])


def test_ffa_search_large_tasks_match_oracle(port):
    """Tasks with up to ~1300 rows run on the cluster path (subtrees through
    L2 scratch); every row above threshold -1e6 is emitted and compared."""
    from gaffa_b200 import core as c
    rng = np.random.default_rng(9)
    n = 300_000
    x = rng.normal(size=n).astype(np.float32)
    tasks, widths = port.make_plan(n, 1e-3, 0.2, 0.6, bins_min=200, bins_max=230)
    want = port.ffa_search(x, tasks, widths, snr_threshold=-1e6)
    got = _search(x, tasks, widths, -1e6)
    assert np.array_equal(got, want)


def test_ffa_peak_buffer_regrows():
    c = core()
    rng = np.random.default_rng(2)
    x = rng.normal(size=50000).astype(np.float32)
    plan = c.make_riptide_ffa_plan(50000, 1e-3, 0.2, 1.0, bins_min=40, bins_max=60)
    prog = c.FfaProgram(plan, max_series=1)
    prog.capacity = 8
    prep = prog.prepare(torch.from_numpy(x).cuda().view(1, -1), 1)
    rec = prog.search(prep, 1, -1e6)
    assert len(rec) > 8 and prog.capacity >= len(rec)


def test_dm_search_block_matches_reference(golden_small):
    """find_dm_peaks on a dedispersed uint32 block (preprocess + FFA + peaks),
    then candidates, bit for bit."""
    c = core()
    g = golden_small
    blk = g["dd_multi"]
    ns = blk.shape[1]
    plan = c.make_riptide_ffa_plan(ns, 1e-3, 0.1, 1.0, bins_min=40, bins_max=64)
    pre = c.PreprocessProgram(ns, 1e-3, window_seconds=0.5, min_points=11, max_series=24)
    ffa = c.FfaProgram(plan, max_series=24)
    t = torch.from_numpy(blk.view(np.int32).copy()).cuda()
    stats = pre.run(t, 24)
    prep = ffa.prepare(t.view(torch.float32), 24, stats)
    peaks = c.sort_peaks(ffa.expand(ffa.search(prep, 24, 5.0), 0, 0.0, 2.5))
    pre.synchronize()
    assert np.array_equal(peaks, g["dm_peaks"])
    assert np.array_equal(c.select_candidates(peaks, ns * 1e-3), g["cands_default"])
    assert np.array_equal(c.select_candidates(peaks, ns * 1e-3, 0.5, 3, False, 5), g["cands_r3_w"])


def test_fold_matches_reference(golden_small):
    c = core()
    g = golden_small
    prof, expo = c.fold_time_series(torch.from_numpy(g["fold_in_u32"].view(np.int32)).cuda(), 0.25, 1e-3, 32)
    np.testing.assert_allclose(prof, g["fold_u32_profile"], rtol=FOLD_RTOL)
    np.testing.assert_allclose(expo, g["fold_u32_exposure"], rtol=1e-12)
    prof, expo = c.fold_time_series(torch.from_numpy(g["pp_scrunched"]).cuda(), 0.1234, 1e-3, 50, 17)
    np.testing.assert_allclose(prof, g["fold_f32_profile"], rtol=FOLD_RTOL, atol=1e-6)
    np.testing.assert_allclose(expo, g["fold_f32_exposure"], rtol=1e-12)


def test_plain_end_to_end_matches_reference(golden_plain):
    """256 ch x 2^18 samples x 512 DMs: dedispersed block digest, raw-peak
    digest and candidate list identical to the reference; fold to 1e-6."""
    from gaffa_b200 import configs, search, synth
    g = golden_plain
    cfg = configs.plain_end_to_end()
    data = synth.generate(cfg.obs)
    assert hashlib.sha256(data.tobytes()).hexdigest() == str(g["input_digest"])
    ds = search.from_config(cfg, dm_batch=128)
    staged = ds.stage(data)
    full = np.concatenate([u32(ds.dedisp.run(staged, b, 128))[:, : ds.nout] for b in range(0, 512, 128)])
    assert full.shape[1] == int(g["nout"])
    assert hashlib.sha256(full.tobytes()).hexdigest() == str(g["dedispersed_digest"])
    res = ds.run(data)
    assert len(res.peaks) == int(g["npeaks"])
    assert np.array_equal(res.peaks[:4096], g["peaks_top"])
    assert hashlib.sha256(res.peaks.tobytes()).hexdigest() == str(g["peaks_digest"])
    assert np.array_equal(res.candidates, g["candidates"])
    np.testing.assert_allclose(res.fold_profile, g["fold_profile"], rtol=FOLD_RTOL)
    h = np.load(Path(__file__).resolve().parent / "golden" / "ref_harmonic.npz")
    assert np.array_equal(res.ranked, h["plain_sorted"])
    assert np.array_equal(res.harmonics, h["plain_rel"])


def test_invalid_arguments_raise_before_launch():
    c = core()
    f = np.linspace(1200.0, 1500.0, 16)
    with pytest.raises(ValueError):
        c.DedispersionProgram(f, 100, 1e-3, 0.0, 1.0, 0)            # ndm == 0
    with pytest.raises(ValueError):
        c.DedispersionProgram(f, 100, 1e-3, 0.0, -1.0, 4)           # dm_step < 0
    with pytest.raises(ValueError):
        c.DedispersionProgram(f, 100, 1e-3, 0.0, 1.0, 4, ref_frequency_mhz=1300.0)
    with pytest.raises(ValueError):
        c.DedispersionProgram(f, 10, 1e-3, 0.0, 1000.0, 4)          # empty output range
    with pytest.raises(ValueError):
        c.make_riptide_ffa_plan(64, 0.25, 0.5, 4.0, bins_min=4, bins_max=5)
    with pytest.raises(RuntimeError):
        c.make_riptide_ffa_plan(64, 0.25, 1.0, 4.0, bins_min=4, bins_max=5, min_periods=2,
                                duty_cycle_max=0.5, max_tasks=1)
    plan = c.make_riptide_ffa_plan(5000, 1e-3, 0.1, 0.5, bins_min=40, bins_max=50)
    with pytest.raises(ValueError):
        c.FfaProgram(plan.with_widths([0]))
    with pytest.raises(ValueError):
        c.FfaProgram(plan.with_widths([40]))
