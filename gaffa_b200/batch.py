"""Batched search of many observations of uneven geometry on one GPU.

The reference searches one observation at a time: one dedispersion launch per
plan (dedispersion_cuda.cu:536-585), then detrend, prepare and one
CudaFfaProgram run per DM tile (cuda_dm_search_benchmark.cpp:179-260).  A
batch of observations with different channel counts, lengths, DM grids and
FFA period ranges would leave the GPU idle at the tail of every launch.
Here a batch is cut into pieces (one observation's contiguous DM range) and
the pieces are packed into waves that fit the series arena.  Each wave runs

* ONE dedispersion launch over all its pieces (gf_dedisp_batch: each CTA
  finds its piece in a block table),
* ONE launch per preprocessing stage (scrunch, running median, detrend,
  statistics) and ONE FFA-prepare launch over all its pieces
  (gf_preprocess_batch, gf_ffa_batch_prepare_all: item tables likewise; the
  prepare folds every octave's downsampling into one pass),
* ONE persistent FFA launch per class over every (piece series, task) item
  of the wave (gf_ffa_batch: the item runs of all members in one table),

captured once into a CUDA graph and replayed on later runs.  The dedispersion
launch shapes (DMs per CTA, channel rows per staging step) come from an
autotuner that times candidate shapes on the observation's own data and
caches the winners by geometry.  Peaks, candidates and harmonic flags are
identical to searching each observation with its own search.DmSearch (the
kernels and the arithmetic are the same, only the launch grouping differs);
the fold of the top candidate agrees to the fold's own tolerance (its FP64
sums are combined by atomics in a run-dependent order).
"""
from __future__ import annotations

import concurrent.futures as cf
import dataclasses
import json
import os
import math
import time
from pathlib import Path

import numpy as np
import torch

from . import _lib, core
from .search import SearchResult


@dataclasses.dataclass
class Piece:
    """DMs [dm_begin, dm_begin + dm_count) of observation obs."""
    obs: int
    dm_begin: int
    dm_count: int


def plan_pieces(ndm: list, bytes_per_dm: list, wave_bytes: int, granularity: int = 8) -> list:
    """Packs every observation's DM range, in observation order, into waves
    of at most wave_bytes, cutting a range where a wave fills up (cuts fall
    on multiples of granularity; a block of granularity DMs larger than a
    wave gets a wave of its own).  Returns [[Piece, ...], ...]."""
    waves, cur, used = [], [], 0
    for i, (n, b) in enumerate(zip(ndm, bytes_per_dm)):
        begin = 0
        while begin < n:
            room = (wave_bytes - used) // b
            cnt = n - begin if n - begin <= room else room // granularity * granularity
            if cnt <= 0:
                if cur:
                    waves.append(cur)
                    cur, used = [], 0
                    continue
                cnt = min(n - begin, granularity)
            cur.append(Piece(i, begin, cnt))
            used += cnt * b
            begin += cnt
    if cur:
        waves.append(cur)
    return waves


class Autotuner:
    """Picks the brute-force dedispersion launch shape (DMs per CTA, channel
    rows per staging step) by timing candidate shapes on a block of the
    observation's highest DMs, and caches the winner by geometry (channels,
    DM step, log2 length) in memory and, given a path, in a JSON file.  All
    shapes give the same sums; only the speed differs."""

    SHAPES = ((8, 64), (8, 32), (8, 16), (4, 32), (4, 16), (2, 16))

    def __init__(self, path: str | Path | None = None, dms: int = 64, repeats: int = 3):
        self.path = Path(path) if path else None
        self.cache = {}
        if self.path is not None and self.path.exists():
            self.cache = json.loads(self.path.read_text())
        self.dms = dms
        self.repeats = repeats
        self.timings = {}

    @staticmethod
    def key(nchans: int, dm_step: float, nsamples: int) -> str:
        return f"brute-u8/nchans={nchans}/dm_step={dm_step:.4g}/log2_nsamples={round(math.log2(nsamples))}"

    def save(self) -> None:
        if self.path is not None:
            self.path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))

    def dedispersion_shape(self, key: str, make_program, staged: torch.Tensor) -> tuple:
        """The cached shape for key, else the fastest of SHAPES on staged
        (make_program(shape) -> DedispersionProgram; shapes whose tiles do
        not fit are skipped)."""
        if key in self.cache:
            return tuple(self.cache[key])
        best, best_ms, trials = None, math.inf, {}
        for shape in self.SHAPES:
            try:
                prog = make_program(shape)
            except ValueError:
                continue
            cnt = min(self.dms, prog.ndm)
            begin = (prog.ndm - cnt) // 8 * 8
            cnt = prog.ndm - begin
            out = torch.empty(cnt * ((prog.nout + 3) // 4 * 4), dtype=torch.int32, device=prog.device)
            prog.run(staged, begin, cnt, out=out)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(self.repeats):
                prog.run(staged, begin, cnt, out=out)
            b.record()
            b.synchronize()
            ms = a.elapsed_time(b) / self.repeats
            trials[f"{shape[0]}x{shape[1]}"] = ms
            if ms < best_ms:
                best, best_ms = shape, ms
        if best is None:
            raise ValueError("no dedispersion launch shape fits this geometry")
        self.timings[key] = trials
        self.cache[key] = list(best)
        self.save()
        return best


class _Wave:
    def __init__(self, pieces):
        self.pieces = pieces
        self.series = []
        self.dd = None
        self.pre = None
        self.ffa = None
        self.graph = None


class BatchSearch:
    """A reusable search of a fixed batch of observations (a list of
    configs.SearchConfig, one per observation; they must share the S/N
    threshold).  run() takes the observations' time-major uint8 filterbanks
    and returns one search.SearchResult per observation."""

    def __init__(self, configs, device_id: int = 0, wave_bytes: int | None = None, tuner: Autotuner | None = None,
                 use_graphs: bool = True, harmonic_options=None, finish_threads: int | None = None):
        self.configs = list(configs)
        if not self.configs:
            raise ValueError("a batch needs at least one observation")
        thr = {c.snr_threshold for c in self.configs}
        if len(thr) != 1:
            raise ValueError("observations of one batch share the S/N threshold")
        for c in self.configs:
            if c.dedispersion != "brute" or c.obs.nbits != 8:
                raise ValueError("batched search takes 8-bit brute-force observations")
        self.snr_threshold = thr.pop()
        # host threads for the per-observation steps after the search
        self.finish_threads = finish_threads or max(1, min(len(self.configs), os.cpu_count() or 1, 16))
        self.device = torch.device("cuda", device_id)
        self.device_id = device_id
        self.use_graphs = use_graphs
        self.tuner = tuner
        self.harmonic_options = harmonic_options if harmonic_options is not None else core.harmonic_options()
        self.dd, self.plans, self.staged, self.strides, self.prep = [], [], [], [], []
        for c in self.configs:
            o = c.obs
            dd = core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm,
                                          device_id=device_id)
            self.staged.append(torch.empty(int(dd.info.staged_bytes), dtype=torch.uint8, device=self.device))
            self.dd.append(dd)
            plan = core.make_riptide_ffa_plan(dd.nout, o.tsamp, c.period_min, c.period_max, bins_min=c.bins_min,
                                              bins_max=c.bins_max, duty_cycle_max=c.duty_cycle_max)
            if c.width_trials is not None:
                plan = plan.with_widths(c.width_trials)
            self.plans.append(plan)
            self.strides.append((dd.nout + 3) // 4 * 4)
            self.prep.append(plan.prepared_floats)
        self._tuned = False
        per_dm = [4 * (s + p) for s, p in zip(self.strides, self.prep)]
        if wave_bytes is None:
            free = torch.cuda.mem_get_info(self.device)[0]
            wave_bytes = max(1 << 28, int(free * 0.4))
        self.wave_bytes = wave_bytes
        self.waves = [_Wave(p) for p in plan_pieces([c.ndm for c in self.configs], per_dm, wave_bytes)]
        biggest = max(sum(pc.dm_count * per_dm[pc.obs] for pc in w.pieces) for w in self.waves)
        self._series_arena = torch.empty(max(4, biggest // 8), dtype=torch.int64, device=self.device)
        max_piece = [0] * len(self.configs)
        for w in self.waves:
            for pc in w.pieces:
                max_piece[pc.obs] = max(max_piece[pc.obs], pc.dm_count)
        self.pre = [core.PreprocessProgram(dd.nout, c.obs.tsamp, window_seconds=c.window_seconds,
                                           min_points=c.min_points, normalise=True, reject_constant=True,
                                           max_series=max(1, m), device_id=device_id)
                    for dd, c, m in zip(self.dd, self.configs, max_piece)]
        self._scratch = None
        self._built = False

    # -- setup --------------------------------------------------------------

    def _tune(self) -> None:
        """Rebuilds each observation's dedispersion program with its tuned
        launch shape (needs the staged data, so it runs on the first run)."""
        for i, c in enumerate(self.configs):
            o = c.obs
            key = Autotuner.key(o.nchans, c.dm_step, o.nsamples)

            def make(shape, o=o, c=c):
                return core.DedispersionProgram(o.frequencies, o.nsamples, o.tsamp, c.dm_low, c.dm_step, c.ndm,
                                                device_id=self.device_id, launch_shape=shape)
            self.dd[i] = make(self.tuner.dedispersion_shape(key, make, self.staged[i]))
        self._tuned = True

    def _build_waves(self) -> None:
        arena = self._series_arena
        for w in self.waves:
            # series first, prepared octaves after them, in one arena shared by all waves
            series, prepared, off = [], [], 0
            for pc in w.pieces:
                n = pc.dm_count * self.strides[pc.obs]
                series.append(arena.view(torch.int32)[off:off + n].view(pc.dm_count, self.strides[pc.obs]))
                off += n
            for pc in w.pieces:
                n = pc.dm_count * self.prep[pc.obs]
                prepared.append(arena.view(torch.float32)[off:off + n].view(pc.dm_count, self.prep[pc.obs]))
                off += n
            w.series = series
            w.dd = core.DedispersionBatch(
                (self.dd[pc.obs], self.staged[pc.obs], pc.dm_begin, pc.dm_count, s, self.strides[pc.obs])
                for pc, s in zip(w.pieces, series))
            w.ffa = core.FfaBatchProgram([(self.plans[pc.obs], pc.dm_count) for pc in w.pieces],
                                         device_id=self.device_id, prepared=prepared, scratch=False)
            # one launch per preprocessing stage and one prepare over every piece
            w.pre = core.PreprocessBatch((self.pre[pc.obs], sr, pc.dm_count) for pc, sr in zip(w.pieces, series))
            w.ffa.bind_series([sr.view(torch.float32) for sr in series],
                              [self.pre[pc.obs].stats[: pc.dm_count] for pc in w.pieces])
            w.graph = None
        need = max(w.ffa.scratch_bytes for w in self.waves)
        self._scratch = torch.empty(max(16, need), dtype=torch.uint8, device=self.device)
        for w in self.waves:
            w.ffa.use_scratch(self._scratch)
        self._built = True

    # -- execution ----------------------------------------------------------

    def _launch_wave(self, w: _Wave) -> None:
        w.dd.run()
        w.pre.run()
        w.ffa.prepare_all()
        w.ffa.search_async(self.snr_threshold)

    def _run_wave(self, w: _Wave) -> None:
        if not self.use_graphs:
            self._launch_wave(w)
            return
        if w.graph is not None:
            w.graph.replay()
            return
        # first run: eager (its results stand), then capture for later runs
        self._launch_wave(w)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch_wave(w)
        w.graph = g

    def _rerun_wave(self, w: _Wave) -> None:
        # the peak buffer grew: the captured graph points at the old one
        w.graph = None
        self._launch_wave(w)

    @property
    def kernel_launches_per_run(self) -> int:
        """Kernels one run launches in its waves: per wave one dedispersion
        launch, three or four preprocessing stages (scrunch, running median,
        detrend, statistics) and one prepare over all its pieces, and one
        FFA launch per class; each observation's fold adds three."""
        if not self._built:
            raise RuntimeError("the waves are built by the first run()")
        return sum(1 + w.pre.kernel_launches + 1 + w.ffa.kernel_launches for w in self.waves)

    def stage(self, filterbanks) -> None:
        """Stages every observation's time-major filterbank (device tensor or
        host array) into the batch's persistent staging buffers."""
        if len(filterbanks) != len(self.configs):
            raise ValueError("one filterbank per observation")
        for dd, fb, st in zip(self.dd, filterbanks, self.staged):
            dd.stage(fb, out=st)

    def run(self, filterbanks=None, timers: dict | None = None) -> list:
        """Searches every observation (filterbanks None: the data staged by
        the last run or stage call)."""
        t0 = time.perf_counter()
        if filterbanks is not None:
            self.stage(filterbanks)
        if self.tuner is not None and not self._tuned:
            self._tune()
        if not self._built:
            self._build_waves()
        t1 = time.perf_counter()
        parts = [[] for _ in self.configs]
        last_wave = {}
        for wi, w in enumerate(self.waves):
            for pc in w.pieces:
                last_wave[pc.obs] = wi
        # An observation's host steps (sort, candidates, harmonics, fold) run
        # on worker threads (the library releases the GIL inside its calls).
        # When every wave replays a captured graph, an observation starts as
        # soon as its last wave is collected, while the next waves run; a run
        # that captures graphs starts them after the last wave, because work
        # from other threads during a capture would invalidate it.
        overlap = not self.use_graphs or all(w.graph is not None for w in self.waves)
        futures = [None] * len(self.configs)
        ready = []
        with cf.ThreadPoolExecutor(max_workers=self.finish_threads) as pool:
            for wi, w in enumerate(self.waves):
                self._run_wave(w)
                rec = w.ffa.collect(self.snr_threshold, rerun=lambda w=w: self._rerun_wave(w))
                peaks, member = w.ffa.expand(rec, [pc.dm_begin for pc in w.pieces],
                                             [self.configs[pc.obs].dm_low for pc in w.pieces],
                                             [self.configs[pc.obs].dm_step for pc in w.pieces])
                for m, pc in enumerate(w.pieces):
                    parts[pc.obs].append(peaks[member == m])
                    if last_wave[pc.obs] == wi:
                        ready.append(pc.obs)
                if overlap:
                    for i in ready:
                        futures[i] = pool.submit(self._finish, i, self.configs[i], parts[i])
                    ready = []
            for i in ready:
                futures[i] = pool.submit(self._finish, i, self.configs[i], parts[i])
            t2 = time.perf_counter()
            for pre in self.pre:
                pre.synchronize()
            for dd in self.dd:
                dd.check()
            results = [f.result() for f in futures]
        t3 = time.perf_counter()
        if timers is not None:
            timers.update(setup=t1 - t0, search=t2 - t1, finish=t3 - t2, total=t3 - t0)
        return results

    def _finish(self, i: int, c, parts) -> SearchResult:
        """Per-observation host steps of DmSearch.run: sort, candidate
        selection, harmonic flagging and the fold of the top candidate."""
        o = c.obs
        peaks = np.concatenate(parts) if parts else np.zeros(0, _lib.PEAK_DTYPE)
        peaks = core.sort_peaks(peaks)
        tobs = o.nsamples * o.tsamp
        cands = core.select_candidates(peaks, tobs, c.frequency_cluster_radius, c.dm_cluster_radius)
        freq = np.asarray(o.frequencies)
        ranked, rel = core.flag_harmonics(cands, tobs, float(freq.min()), float(freq.max()), self.harmonic_options)
        unique = core.remove_harmonics(ranked, rel)
        prof = expo = None
        dd = self.dd[i]
        if len(cands):
            dm_index, period = int(cands[0]["dm_index"]), float(cands[0]["period"])
            b0 = dm_index // 8 * 8
            cnt = min(8, c.ndm - b0)
            series = dd.run(self.staged[i], b0, cnt, out_stride=self.strides[i])
            dd.check()
            prof, expo = core.fold_time_series(series[dm_index - b0, : dd.nout], period, o.tsamp, c.fold_nbin)
        return SearchResult(peaks=peaks, candidates=cands, fold_profile=prof, fold_exposure=expo, nout=dd.nout,
                            ndm=c.ndm, timings={}, gpu_launches=0, ranked=ranked, harmonics=rel,
                            unique_candidates=unique)
