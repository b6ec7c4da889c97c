"""Batched search of uneven observations (gaffa_b200/batch.py).

The batch path regroups launches only: one dedispersion launch per wave, one
persistent FFA launch per class over every observation of the wave, CUDA
graph replays and autotuned dedispersion shapes.  So its results must equal,
bit for bit, the per-observation search (search.DmSearch) whose kernels are
pinned to the reference elsewhere; the dedispersion of a batch is also
checked against the C restatement directly.
"""
import json

import numpy as np
import pytest

from gaffa_b200 import configs
from gaffa_b200.batch import Autotuner, Piece, plan_pieces


def small_batch(nobs=4, seed=7):
    """The batched-uneven laws at test size: 128-512 channels, 2^15-2^17
    samples, 24-96 DMs over 0-300."""
    return configs.batched_uneven(seed=seed, nobs=nobs, nchans_choices=(128, 256, 512), log2_nsamples=(15.0, 17.0),
                                  ndm_range=(24, 96), dm_max=300.0)


# ---------------------------------------------------------------------------
# host logic (no GPU)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("ndm,bpd,budget", [([20, 100, 7], [10, 10, 10], 400), ([20], [1000], 400),
                                             ([37, 5, 64, 100], [12, 40, 8, 16], 1000),
                                             ([300], [4], 10**9)])
def test_plan_pieces_cover_every_dm_once(ndm, bpd, budget):
    waves = plan_pieces(ndm, bpd, budget)
    for i, n in enumerate(ndm):
        pieces = sorted((p for w in waves for p in w if p.obs == i), key=lambda p: p.dm_begin)
        assert pieces[0].dm_begin == 0
        for a, b in zip(pieces, pieces[1:]):
            assert a.dm_begin + a.dm_count == b.dm_begin
        assert pieces[-1].dm_begin + pieces[-1].dm_count == n
        assert all(p.dm_begin % 8 == 0 and p.dm_count > 0 for p in pieces)
    for w in waves:
        used = sum(p.dm_count * bpd[p.obs] for p in w)
        # over budget only for a lone block of 8 DMs
        assert used <= budget or (len(w) == 1 and w[0].dm_count <= 8)


def test_plan_pieces_keeps_small_batches_in_one_wave():
    assert plan_pieces([16, 24], [4, 4], 10**6) == [[Piece(0, 0, 16), Piece(1, 0, 24)]]


def test_batched_uneven_follows_its_laws():
    cs = configs.batched_uneven()
    assert len(cs) == 64
    for c in cs:
        o = c.obs
        assert o.nchans in (1024, 2048, 4096) and o.nbits == 8 and o.tsamp == 64e-6
        assert 2 ** 20 - 16 <= o.nsamples <= 2 ** 23 + 16
        assert 256 <= c.ndm <= 4096
        assert 0.1 <= c.period_min < c.period_max <= 10.0
        assert 0 <= len(o.pulsars) <= 4
        assert abs(c.dm_low + (c.ndm - 1) * c.dm_step - 1000.0) < 1e-9
    assert len({c.obs.seed for c in cs}) == 64


def test_autotuner_uses_its_cache(tmp_path):
    path = tmp_path / "tune.json"
    key = Autotuner.key(512, 0.5, 1 << 17)
    path.write_text(json.dumps({key: [4, 32]}))
    t = Autotuner(path)

    def never(shape):
        raise AssertionError("a cached shape must not be re-measured")
    assert t.dedispersion_shape(key, never, None) == (4, 32)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
def test_dedisp_batch_matches_single_launches_and_oracle(port):
    torch = _cuda()
    from gaffa_b200 import core
    cs = small_batch(3, seed=1)
    progs, staged, host = [], [], []
    for c in cs:
        o = c.obs
        p = core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm)
        x = core.synth_generate(o)
        progs.append(p)
        staged.append(p.stage(x))
        host.append(x)
    # uneven pieces: a middle range, a whole grid, a tail
    ranges = [(8, cs[0].ndm - 8 - 3), (0, cs[1].ndm), (cs[2].ndm // 16 * 8, cs[2].ndm - cs[2].ndm // 16 * 8)]
    outs, items = [], []
    for p, s, (b0, cnt) in zip(progs, staged, ranges):
        stride = (p.nout + 3) // 4 * 4 + 4
        out = torch.full((cnt * stride,), -1, dtype=torch.int32, device="cuda")
        outs.append((out, stride))
        items.append((p, s, b0, cnt, out, stride))
    batch = core.DedispersionBatch(items)
    batch.run()
    torch.cuda.synchronize()
    for i, (p, s, (b0, cnt)) in enumerate(zip(progs, staged, ranges)):
        out, stride = outs[i]
        got = out.view(cnt, stride)[:, : p.nout].cpu().numpy().view(np.uint32)
        want = p.run(s, b0, cnt)[:, : p.nout].cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want)
    # the first item against the C restatement
    c = cs[0]
    freq = np.asarray(c.obs.frequencies, np.float64)
    ref = port.dedisperse_multi_dm(host[0].cpu().numpy(), freq, c.dm_low, c.dm_step, c.ndm, float(freq.max()),
                                   c.obs.tsamp)
    out, stride = outs[0]
    b0, cnt = ranges[0]
    got = out.view(cnt, stride)[:, : progs[0].nout].cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref[b0:b0 + cnt])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(8, 64), (4, 32), (2, 16), (1, 8), (8, 8)])
def test_dedispersion_launch_shapes_give_identical_sums(shape):
    torch = _cuda()
    from gaffa_b200 import core
    c = small_batch(1, seed=3)[0]
    o = c.obs
    x = core.synth_generate(o)
    base = core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm)
    st = base.stage(x)
    want = base.run(st)[:, : base.nout].cpu()
    p = core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm,
                                 launch_shape=shape)
    assert torch.equal(p.run(st)[:, : p.nout].cpu(), want)


@pytest.mark.gpu
def test_dedispersion_rejects_bad_launch_shapes():
    _cuda()
    from gaffa_b200 import core
    c = small_batch(1, seed=3)[0]
    o = c.obs
    for shape in ((3, 64), (8, 48), (1, 64)):          # not a shape; not a chunk size; tile too large
        with pytest.raises(ValueError):
            core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm,
                                     launch_shape=shape)


def _records_key(rec, task_offset=0):
    return sorted((int(r["task"]) + task_offset, int(r["series"]), int(r["shift"]), int(r["phase"]),
                   int(r["width_index"]), float(r["snr"])) for r in rec)


@pytest.mark.gpu
def test_ffa_batch_matches_one_program_per_plan():
    torch = _cuda()
    from gaffa_b200 import core
    gen = torch.Generator(device="cuda").manual_seed(5)
    specs = [(40_000, 64e-6, 0.05, 1.0, 3), (131_072, 64e-6, 0.2, 4.0, 5), (70_001, 128e-6, 0.5, 4.0, 2)]
    plans, series = [], []
    for n, ts, p0, p1, ns in specs:
        plans.append(core.make_riptide_ffa_plan(n, ts, p0, p1, bins_min=48, bins_max=80, duty_cycle_max=0.1))
        series.append(torch.randn((ns, n), generator=gen, device="cuda"))
    batch = core.FfaBatchProgram([(pl, s.shape[0]) for pl, s in zip(plans, series)])
    stats = []
    for m, (pl, s) in enumerate(zip(plans, series)):
        st = torch.zeros((s.shape[0], 2), dtype=torch.float64, device="cuda")
        st[:, 1] = 1.0
        stats.append(st)
        batch.prepare(m, s, st)
        assert batch.member_info[m].prepared_floats == pl.prepared_floats
    batch.search_async(3.0)
    got = batch.collect(3.0)
    assert len(got) > 0
    want = []
    for m, (pl, s, st) in enumerate(zip(plans, series, stats)):
        prog = core.FfaProgram(pl, max_series=s.shape[0])
        assert prog.prepared_floats == pl.prepared_floats
        prep = prog.prepare(s, s.shape[0], st)
        mi = batch.member_info[m]
        want += _records_key(prog.search(prep, s.shape[0], 3.0), int(mi.task_begin))
        # expansion per member equals the single program's
        mine = got[(got["task"] >= mi.task_begin) & (got["task"] < mi.task_begin + mi.ntasks)]
        peaks, member = batch.expand(mine, [0, 0, 0], [0.0, 0.0, 0.0], [1.0, 1.0, 1.0])
        assert (member == m).all()
        local = mine.copy()
        local["task"] -= mi.task_begin
        ref = prog.expand(local, 0, 0.0, 1.0)
        order = ["dm_index", "period", "phase", "width"]
        assert np.array_equal(np.sort(peaks, order=order), np.sort(ref, order=order))
    assert _records_key(got) == sorted(want)


@pytest.mark.gpu
def test_preprocess_batch_and_prepare_all_match_single_launches():
    """One launch per preprocessing stage over series sets of different
    lengths, windows (scrunched and exact medians) and input types, and one
    prepare over every member, equal the per-set launches bit for bit."""
    torch = _cuda()
    from gaffa_b200 import core
    gen = torch.Generator(device="cuda").manual_seed(9)
    # (nsamples, tsamp, window_seconds, min_points, nseries, uint32 input)
    specs = [(40_000, 64e-6, 0.05, 101, 3, True), (131_072, 64e-6, 1.0, 101, 5, True),
             (70_001, 128e-6, 0.1, 51, 2, False), (9_000, 64e-6, 0.02, 301, 4, True)]
    pres, bufs, want = [], [], []
    for n, ts, win, mp, ns, u32 in specs:
        pre = core.PreprocessProgram(n, ts, window_seconds=win, min_points=mp, max_series=ns)
        stride = (n + 3) // 4 * 4 + 4
        if u32:
            x = torch.randint(0, 60_000, (ns, stride), generator=gen, device="cuda", dtype=torch.int32)
        else:
            x = torch.randn((ns, stride), generator=gen, device="cuda") * 3.0 + 7.0
        ref = x.clone()
        stats = pre.run(ref, ns).clone()
        pre.synchronize()
        want.append((ref[:, :n].clone(), stats))
        pres.append(pre)
        bufs.append(x)
    assert any(int(p.info.scrunch_factor) > 1 for p in pres) and any(int(p.info.scrunch_factor) == 1 for p in pres)
    batch = core.PreprocessBatch((p, b, spec[4]) for p, b, spec in zip(pres, bufs, specs))
    batch.run()
    for p in pres:
        p.synchronize()
    for (n, *_), b, p, (ref, stats) in zip(specs, bufs, pres, want):
        assert torch.equal(b[:, :n], ref)
        assert torch.equal(p.stats[: b.shape[0]], stats)
    # the prepared FFA inputs of every member in one launch
    plans = [core.make_riptide_ffa_plan(n, ts, 0.05, 0.5, bins_min=48, bins_max=80, duty_cycle_max=0.1)
             for n, ts, *_ in specs]
    one = core.FfaBatchProgram([(pl, spec[4]) for pl, spec in zip(plans, specs)])
    two = core.FfaBatchProgram([(pl, spec[4]) for pl, spec in zip(plans, specs)])
    for t in one.prepared + two.prepared:
        t.zero_()  # padding between octaves is never written
    views = [b.view(torch.float32) for b in bufs]
    for m, (v, p) in enumerate(zip(views, pres)):
        one.prepare(m, v, p.stats[: v.shape[0]])
    two.bind_series(views, [p.stats[: v.shape[0]] for v, p in zip(views, pres)])
    two.prepare_all()
    torch.cuda.synchronize()
    for a, b, mi in zip(one.prepared, two.prepared, one.member_info):
        k = int(mi.nseries) * int(mi.prepared_floats)
        assert torch.equal(a.reshape(-1)[:k], b.reshape(-1)[:k])


def _assert_same_result(a, b):
    assert np.array_equal(a.peaks, b.peaks)
    assert np.array_equal(a.candidates, b.candidates)
    assert np.array_equal(a.unique_candidates, b.unique_candidates)
    if a.fold_profile is None:
        assert b.fold_profile is None
    else:
        # the fold's FP64 sums are combined by shared-memory atomics, in a
        # run-dependent order (the parity tests' fold tolerance)
        np.testing.assert_allclose(np.asarray(a.fold_profile), np.asarray(b.fold_profile), rtol=1e-6)
        np.testing.assert_allclose(np.asarray(a.fold_exposure), np.asarray(b.fold_exposure), rtol=1e-12)


@pytest.mark.gpu
def test_batch_search_matches_per_observation_search(tmp_path):
    _cuda()
    from gaffa_b200 import batch, core, search
    cs = small_batch(4, seed=11)
    for c in cs:
        c.snr_threshold = 6.0
    data = [core.synth_generate(c.obs) for c in cs]
    want = [search.from_config(c).run(x) for c, x in zip(cs, data)]
    assert sum(len(w.peaks) for w in want) > 0
    # a small arena: several waves, observations cut across waves
    per_dm = max(8 * c.obs.nsamples for c in cs)
    bs = batch.BatchSearch(cs, wave_bytes=per_dm * 40, tuner=batch.Autotuner(tmp_path / "tune.json"))
    assert len(bs.waves) > 1
    first = bs.run(data)
    for a, b in zip(first, want):
        _assert_same_result(a, b)
    # replays of the captured graphs, on the data staged into the same buffers
    again = bs.run(data)
    for a, b in zip(again, want):
        _assert_same_result(a, b)
    assert all(w.graph is not None for w in bs.waves)
    assert json.loads((tmp_path / "tune.json").read_text())


@pytest.mark.gpu
def test_batch_search_peak_buffer_growth_and_eager_mode():
    _cuda()
    from gaffa_b200 import batch, core, search
    cs = small_batch(2, seed=13)
    for c in cs:
        c.snr_threshold = 3.0          # many peaks: the 65536-record buffer overflows
    data = [core.synth_generate(c.obs) for c in cs]
    want = [search.from_config(c).run(x) for c, x in zip(cs, data)]
    bs = batch.BatchSearch(cs, use_graphs=True)
    got = bs.run(data)
    for a, b in zip(got, want):
        _assert_same_result(a, b)
    assert any(w.ffa.capacity > (1 << 16) for w in bs.waves)
    got = bs.run(data)          # captured again after the buffer grew
    for a, b in zip(got, want):
        _assert_same_result(a, b)
    plain = batch.BatchSearch(cs, use_graphs=False).run(data)
    for a, b in zip(plain, want):
        _assert_same_result(a, b)


@pytest.mark.gpu
def test_run_many_overlaps_staging_and_matches_run():
    """DmSearch.run_many stages observation i + 1 on a helper thread and side
    stream while observation i is searched; every result equals run()."""
    _cuda()
    import dataclasses
    from gaffa_b200 import search, synth
    c = small_batch(1, seed=5)[0]
    c.snr_threshold = 6.0
    hosts = [synth.generate(dataclasses.replace(c.obs, seed=c.obs.seed + k)) for k in range(3)]
    ds = search.from_config(c)
    want = [ds.run(h) for h in hosts]
    got = ds.run_many(hosts)
    assert len(got) == 3
    for a, b in zip(got, want):
        _assert_same_result(a, b)
    assert sum(len(r.peaks) for r in got) > 0
