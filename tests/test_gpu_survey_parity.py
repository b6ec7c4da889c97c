"""Parity at the benchmarked configuration and against the FP64 oracle.

* The survey-size observation the bench times (4096 channels x 2^23 samples,
  2048 DM trials over 0-1000, FFA 0.1-10 s, 8 injected pulsars) runs through
  DmSearch exactly as the bench runs it.  For sampled DM trials -- the first
  and last of each DM batch among them -- the dedispersed rows must equal the
  reference's dedisperse_multi_dm_cpu bit for bit, each trial's raw peaks must
  equal the reference's find_dm_peaks_cpu (dm_search.cpp:142-199) byte for
  byte, and the candidates selected from those peaks must be identical.
* The survey plan's largest FFA tasks (5348 rows x 180 bins and the largest
  of every bin class, three column passes with the remainder last) run on
  the CUDA search and are compared with the C restatement of the FFA
  (ffa.cpp:173-195, ffa_detection.cpp:126-170), every row and width.
* CUDA S/N of every evaluated row and width of a plain-workload plan is
  within 1e-5 relative of the FP64 restatement (oracle/ffa64_oracle.c).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-5          # relative for |S/N| >= 1, absolute below


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cpu_checker():
    """The reference's own CPU sources when built, else the C restatement."""
    from oracle.oracle import Oracle
    return Oracle("reference" if Oracle.available("reference") else "port")


def _search_all_rows(series, tasks, widths):
    """CUDA search of one series with no effective threshold: one peak per
    (task, evaluated row, width), as records (task, shift, width_index, snr)."""
    from gaffa_b200 import core as c
    plan = c.FfaPlan(tasks, widths)
    prog = c.FfaProgram(plan, max_series=1)   # the peak buffer grows and the search re-runs on overflow
    s = torch.from_numpy(np.ascontiguousarray(series, np.float32)).cuda().view(1, -1)
    prep = prog.prepare(s, 1)
    return prog, prog.search(prep, 1, -1e30)


def test_cuda_snr_within_1e5_of_fp64_oracle(port):
    """Plain-workload plan (periods 0.2-2 s, 64 us, widths 1..32) on a
    normalised 2^18-sample series with a weak pulse; every task, every row,
    every width."""
    from oracle import oracle
    n, tsamp = 1 << 18, 64e-6
    rng = np.random.default_rng(17)
    x = rng.normal(size=n).astype(np.float32)
    ph = (np.arange(n) * tsamp / 0.5) % 1.0
    x += (0.6 * np.exp(-0.5 * ((ph - 0.3) / 0.004) ** 2)).astype(np.float32)
    x = ((x - x.mean()) / x.std()).astype(np.float32)
    tasks, _ = port.make_plan(n, tsamp, 0.2, 2.0)
    widths = np.array([1, 2, 4, 8, 16, 32], np.uint64)
    _, rec = _search_all_rows(x, tasks, widths)
    assert len(rec) == int(tasks["rows_eval"].sum()) * len(widths)
    worst = 0.0
    for ti in range(len(tasks)):
        r = rec[rec["task"] == ti]
        s64, _ = oracle.ffa64_task_snr(x, tasks[ti], widths)
        got = np.full(s64.shape, np.nan)
        got[r["shift"].astype(int), r["width_index"].astype(int)] = r["snr"]
        err = np.abs(got - s64) / np.maximum(1.0, np.abs(s64))
        worst = max(worst, float(np.nanmax(err)))
        assert not np.isnan(got).any()
    assert worst <= SNR_RTOL, worst


def test_survey_plan_largest_tasks_match_restatement(port):
    """The survey plan (8,357,464 samples, 64 us, 0.1-10 s, duty <= 0.1): its
    largest task (5348 rows x 180 bins, split into subtrees and three column
    passes), the largest task of every bin class and the last task of each of
    the first octaves, every row and width, bit for bit."""
    from gaffa_b200 import configs
    cfg = configs.survey_size()
    n = 8_357_464
    tasks, widths = port.make_plan(n, cfg.obs.tsamp, cfg.period_min, cfg.period_max,
                                   duty_cycle_max=cfg.duty_cycle_max)
    pick = {int(np.argmax(tasks["rows"]))}
    nb = (tasks["bins"].astype(int) + 31) // 32
    for k in np.unique(nb):
        idx = np.flatnonzero(nb == k)
        pick.add(int(idx[np.argmax(tasks["rows"][idx] * tasks["bins"][idx])]))
    factors = np.unique(tasks["downsample_factor"])
    for f in factors[:3]:
        pick.add(int(np.flatnonzero(tasks["downsample_factor"] == f)[-1]))
    sel = np.ascontiguousarray(tasks[sorted(pick)])
    assert int(sel["rows"].max()) == 5348
    rng = np.random.default_rng(23)
    x = rng.normal(size=n).astype(np.float32)
    from gaffa_b200 import core as c
    prog, rec = _search_all_rows(x, sel, widths)
    got = c.sort_peaks(prog.expand(rec))
    want = port.ffa_search(x, sel, widths, snr_threshold=-1e30)
    assert len(got) == len(want) == int(sel["rows_eval"].sum()) * len(widths)
    assert np.array_equal(got, want)


def test_survey_size_observation_matches_reference_on_sampled_dms():
    """The benchmarked observation end to end through DmSearch; sampled DM
    trials checked against the reference CPU path."""
    psutil = pytest.importorskip("psutil")
    from gaffa_b200 import configs, core, search
    cfg = configs.survey_size()
    obs = cfg.obs
    need = obs.nsamples * obs.nchans * 1.3
    if psutil.virtual_memory().available < need:
        pytest.skip("not enough host memory for a host copy of the survey-size filterbank")
    raw = core.synth_generate(obs)
    ds = search.from_config(cfg)
    res = ds.run(raw)
    assert ds.dm_batch % 8 == 0 and ds.dm_batch < cfg.ndm
    nout = ds.nout
    b = ds.dm_batch
    sample = sorted({0, b - 1, b, 2 * b - 1, 2 * b, 1023, 1800, cfg.ndm - 1} & set(range(cfg.ndm)))
    assert len(sample) >= 8
    # the GPU's dedispersed rows of the sampled trials (groups of 8 from the staged input)
    staged = ds.stage(raw)
    rows = {}
    for dm in sample:
        g0 = dm // 8 * 8
        blk = ds.dedisp.run(staged, g0, min(8, cfg.ndm - g0))
        rows[dm] = blk[dm - g0, :nout].cpu().numpy().view(np.uint32).copy()
    del staged
    host = raw.cpu().numpy()
    del raw
    torch.cuda.empty_cache()
    ref = _cpu_checker()
    want = np.stack([ref.dedisperse_multi_dm(host, obs.frequencies, cfg.dm_low + dm * cfg.dm_step, cfg.dm_step, 1,
                                             obs.ref_frequency, obs.tsamp)[0, :nout] for dm in sample])
    del host
    got = np.stack([rows[dm] for dm in sample])
    for i, dm in enumerate(sample):
        assert np.array_equal(got[i], want[i]), f"dedispersed row of DM trial {dm} differs"
    dms = cfg.dms[sample]
    widths = None if cfg.width_trials is None else np.array(cfg.width_trials, np.uint64)
    ref_peaks = ref.find_dm_peaks(np.ascontiguousarray(want), dms, obs.tsamp, cfg.plan_options(),
                                  cfg.preprocess_options(), cfg.snr_threshold, widths=widths)
    # the reference numbers the trials of its block 0..len(sample)-1
    ref_peaks["dm_index"] = np.asarray(sample, np.uint64)[ref_peaks["dm_index"].astype(int)]
    mine = res.peaks[np.isin(res.peaks["dm_index"], np.asarray(sample, np.uint64))]
    assert len(mine) == len(ref_peaks) and len(mine) > 0
    for dm in sample:
        a = mine[mine["dm_index"] == dm]
        w = ref_peaks[ref_peaks["dm_index"] == dm]
        assert np.array_equal(a, w), f"raw peaks of DM trial {dm} differ ({len(a)} vs {len(w)})"
    assert np.array_equal(mine, ref_peaks)
    tobs = obs.nsamples * obs.tsamp
    assert np.array_equal(core.select_candidates(mine, tobs), ref.select_candidates(ref_peaks, tobs))
