"""The DM-search pipeline on one GPU: filterbank -> dedispersion -> detrend +
normalise -> per-octave downsampling + FFA + boxcar S/N -> peaks ->
candidates -> harmonic flagging -> fold of the best candidate.

This is the chain the reference wires up in
benchmarks/cuda_dm_search_benchmark.cpp:179-260 (plus select_candidates_cpu
and fold_time_series_cpu), built on the device programs of core.py.  The
filterbank is staged once; DM trials are processed in batches so the
dedispersed block, the prepared octaves and the FFA scratch stay within a
fixed memory budget.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np
import torch

from . import _lib, core


@dataclasses.dataclass
class SearchResult:
    peaks: np.ndarray            # PEAK_DTYPE, sorted by is_better_dm_peak
    candidates: np.ndarray       # CAND_DTYPE
    fold_profile: np.ndarray | None
    fold_exposure: np.ndarray | None
    nout: int
    ndm: int
    timings: dict
    gpu_launches: int = 0
    # flag_harmonics_cpu of the candidates (harmonic.cpp:245-292): ranked
    # candidates and their relations (HARMONIC_DTYPE), then the survivors
    ranked: np.ndarray | None = None
    harmonics: np.ndarray | None = None
    unique_candidates: np.ndarray | None = None
    # raw peaks found; equals len(peaks) unless candidates were selected on the
    # device, where the raw peaks stay on the device and `peaks` is empty
    peak_count: int = 0

    @property
    def dm_trial_samples(self) -> int:
        return self.ndm * self.nout


class _StageTimer:
    """Records CUDA events around a stage's launches into timers[name]."""

    def __init__(self, timers, name):
        self.timers, self.name = timers, name

    def __enter__(self):
        if self.timers is not None:
            self.a = torch.cuda.Event(enable_timing=True)
            self.a.record()
        return self

    def __exit__(self, *exc):
        if self.timers is not None:
            b = torch.cuda.Event(enable_timing=True)
            b.record()
            self.timers.setdefault(self.name, []).append((self.a, b))


class DmSearch:
    """A reusable search for one observation geometry and set of options."""

    def __init__(self, frequency_mhz, nsamples: int, tsamp: float, dm_low: float, dm_step: float, ndm: int,
                 period_min: float, period_max: float, bins_min: int = 180, bins_max: int = 256,
                 duty_cycle_max: float = 0.2, width_trials=None, window_seconds: float = 1.0,
                 min_points: int = 101, snr_threshold: float = 8.0, nbits: int = 8,
                 algorithm: str = "brute", subband_channels: int = 32, ndm_per_nominal: int = 32,
                 frequency_cluster_radius: float = 0.1, dm_cluster_radius: int = 1, fold_nbin: int = 64,
                 dm_batch: int | None = None, memory_budget: int | None = None, device_id: int = 0,
                 harmonic_options=None, launch_shape: tuple[int, int] | None = None,
                 device_candidates: bool = False, peak_capacity: int | None = None):
        """device_candidates: keep the raw peak records on the device and select
        candidates there (gf_select_candidates_device) -- for workloads with
        10^7 or more raw peaks, whose host expansion and sort would dominate;
        the result's `peaks` is then empty and `peak_count` counts them.
        peak_capacity: initial peak-record capacity per DM batch (it grows and
        the batch is re-searched when exceeded)."""
        self.device = torch.device("cuda", device_id)
        freq = np.asarray(frequency_mhz, dtype=np.float64)
        self.frequency_low_mhz, self.frequency_high_mhz = float(freq.min()), float(freq.max())
        self.harmonic_options = harmonic_options if harmonic_options is not None else core.harmonic_options()
        self.nsamples, self.tsamp = nsamples, tsamp
        self.dm_low, self.dm_step, self.ndm = dm_low, dm_step, ndm
        self.snr_threshold = snr_threshold
        self.frequency_cluster_radius = frequency_cluster_radius
        self.dm_cluster_radius = dm_cluster_radius
        self.fold_nbin = fold_nbin
        self.dedisp = core.DedispersionProgram(frequency_mhz, nsamples, tsamp, dm_low, dm_step, ndm, nbits=nbits,
                                               algorithm=algorithm, subband_channels=subband_channels,
                                               ndm_per_nominal=ndm_per_nominal, device_id=device_id,
                                               launch_shape=launch_shape if algorithm == "brute" else None)
        self.nout = self.dedisp.nout
        plan = core.make_riptide_ffa_plan(self.nout, tsamp, period_min, period_max, bins_min=bins_min,
                                          bins_max=bins_max, duty_cycle_max=duty_cycle_max)
        if width_trials is not None:
            plan = plan.with_widths(width_trials)
        self.plan = plan
        self.out_stride = ((self.nout + 3) // 4) * 4
        g = self.dedisp.batch_granularity
        if dm_batch is None:
            free = torch.cuda.mem_get_info(self.device)[0] if memory_budget is None else memory_budget
            per_dm = self.out_stride * 4 + plan.prepared_floats * 4
            budget = int(free * 0.45) - self.dedisp.info.staged_bytes - (1 << 30)
            dm_batch = max(g, min(ndm, budget // max(1, per_dm)))
        dm_batch = max(g, (dm_batch // g) * g)
        self.dm_batch = min(dm_batch, ((ndm + g - 1) // g) * g)
        self.pre = core.PreprocessProgram(self.nout, tsamp, window_seconds=window_seconds, min_points=min_points,
                                          normalise=True, reject_constant=True, max_series=self.dm_batch,
                                          device_id=device_id)
        self.ffa = core.FfaProgram(plan, max_series=self.dm_batch, device_id=device_id)
        self.device_candidates = device_candidates
        if peak_capacity is not None and peak_capacity > self.ffa.capacity:
            self.ffa.capacity = int(peak_capacity)
            self.ffa.peaks = torch.empty(self.ffa.capacity * 24, dtype=torch.uint8, device=self.device)
        self._series = torch.empty(self.dm_batch * self.out_stride, dtype=torch.int32, device=self.device)
        self._prepared = torch.empty((self.dm_batch, self.ffa.prepared_floats), dtype=torch.float32,
                                     device=self.device)
        self._workspace = None
        if algorithm == "subband":
            self._workspace = torch.empty(self.dedisp.workspace_bytes(self.dm_batch), dtype=torch.uint8,
                                          device=self.device)

    def stage(self, filterbank) -> torch.Tensor:
        return self.dedisp.stage(filterbank)

    def batches(self, dm_ranges=None):
        """(first DM, count) of every batch; dm_ranges (optional) restricts the
        search to [begin, end) ranges of DM indices, begin a multiple of the
        dedispersion granularity."""
        ranges = [(0, self.ndm)] if dm_ranges is None else dm_ranges
        g = self.dedisp.batch_granularity
        for begin, end in ranges:
            if begin % g or not 0 <= begin < end <= self.ndm:
                raise ValueError(f"DM range ({begin}, {end}) must start at a multiple of {g} within [0, ndm]")
            for b0 in range(begin, end, self.dm_batch):
                yield b0, min(self.dm_batch, end - b0)

    def search_staged(self, staged: torch.Tensor, timers: dict | None = None, dm_ranges=None) -> tuple:
        """Runs every DM batch (or the batches of dm_ranges); returns (raw
        peaks, kernel launches).

        timers (optional) collects CUDA events around each stage's launches:
        dedisperse, preprocess, prepare, ffa."""
        parts = []
        launches = 0
        dd_kernels = 1 if self.dedisp.algorithm == "brute" else 2
        ffa_kernels = self.ffa.kernel_launches
        for b0, cnt in self.batches(dm_ranges):
            with _StageTimer(timers, "dedisperse"):
                dd = self.dedisp.run(staged, b0, cnt, out=self._series, out_stride=self.out_stride,
                                     workspace=self._workspace)
            with _StageTimer(timers, "preprocess"):
                stats = self.pre.run(dd, cnt)
            with _StageTimer(timers, "prepare"):
                self.ffa.prepare(dd.view(torch.float32), cnt, stats, out=self._prepared)
            with _StageTimer(timers, "ffa"):
                self.ffa.search_async(self._prepared, cnt, self.snr_threshold)
            if self.device_candidates:
                n = self.ffa.count(self._prepared, cnt, self.snr_threshold)
                parts.append((self.ffa.peaks[: n * 24].clone(), n, b0))
            else:
                rec = self.ffa.collect(self._prepared, cnt, self.snr_threshold)
                parts.append(self.ffa.expand(rec, b0, self.dm_low, self.dm_step))
            launches += dd_kernels + 4 + 1 + ffa_kernels
        self.pre.synchronize()
        self.dedisp.check()
        if self.device_candidates:
            return parts, launches
        peaks = np.concatenate(parts) if parts else np.zeros(0, _lib.PEAK_DTYPE)
        return peaks, launches

    def _device_candidates(self, parts, tobs: float) -> tuple[np.ndarray, int]:
        """Candidates of the device-resident records of every batch."""
        segments, at = [], 0
        for _, n, b0 in parts:
            segments.append((at, n, b0))
            at += n
        if at == 0:
            return np.zeros(0, _lib.CAND_DTYPE), 0
        records = torch.cat([r for r, _, _ in parts]) if len(parts) > 1 else parts[0][0]
        cands = core.select_candidates_device(self.ffa, records, segments, self.dm_low, self.dm_step, tobs,
                                              self.frequency_cluster_radius, self.dm_cluster_radius)
        return cands, at

    def fold_candidate(self, staged: torch.Tensor, dm_index: int, period: float):
        """fold_time_series of the candidate's uint32 dedispersed series."""
        g = self.dedisp.batch_granularity
        b0 = (dm_index // g) * g
        cnt = min(g, self.ndm - b0)
        ws = None
        if self.dedisp.algorithm == "subband":
            ws = torch.empty(self.dedisp.workspace_bytes(cnt), dtype=torch.uint8, device=self.device)
        dd = self.dedisp.run(staged, b0, cnt, out_stride=self.out_stride, workspace=ws)
        self.dedisp.check()
        row = dd[dm_index - b0, : self.nout]
        return core.fold_time_series(row, period, self.tsamp, self.fold_nbin)

    def run(self, filterbank, observation_seconds: float | None = None, timers: dict | None = None,
            dm_ranges=None) -> SearchResult:
        t0 = time.perf_counter()
        with _StageTimer(timers, "stage"):
            staged = self.stage(filterbank)
        torch.cuda.synchronize(self.device)
        return self._search(staged, t0, observation_seconds, timers, dm_ranges)

    def run_many(self, filterbanks, observation_seconds: float | None = None) -> list:
        """Searches observations one after another (host arrays or pinned host
        tensors, time-major).  A helper thread stages observation i + 1 into a
        second staging buffer (host-to-device copies and the transpose, on a
        side stream) while observation i is searched, so the copies hide behind
        the search.  Results equal run() of each observation."""
        import threading
        filterbanks = list(filterbanks)
        n = len(filterbanks)
        bufs = [torch.empty(int(self.dedisp.info.staged_bytes), dtype=torch.uint8, device=self.device)
                for _ in range(min(2, n))]
        side = torch.cuda.Stream(self.device)
        ready = [threading.Event() for _ in range(n)]
        freed = [threading.Event() for _ in range(n)]
        errors = []

        def stage_all():
            try:
                torch.cuda.set_device(self.device)
                for i, fb in enumerate(filterbanks):
                    if i >= 2:
                        freed[i - 2].wait()
                        if errors:
                            return
                    with torch.cuda.stream(side):
                        self.dedisp.stage(fb, stream=side, out=bufs[i % 2])
                    side.synchronize()
                    ready[i].set()
            except Exception as exc:  # re-raised on the searching thread
                errors.append(exc)
                for e in ready:
                    e.set()

        worker = threading.Thread(target=stage_all, daemon=True)
        worker.start()
        results = []
        try:
            for i in range(n):
                t0 = time.perf_counter()
                ready[i].wait()
                if errors:
                    raise errors[0]
                results.append(self._search(bufs[i % 2], t0, observation_seconds, None, None))
                torch.cuda.synchronize(self.device)
                freed[i].set()
        finally:
            if len(results) < n:
                # stop the helper before it stages into a buffer still in use
                errors.append(RuntimeError("search stopped"))
                for e in freed:
                    e.set()
            worker.join()
        return results

    def _search(self, staged: torch.Tensor, t0: float, observation_seconds, timers, dm_ranges) -> SearchResult:
        t = {}
        t1 = time.perf_counter()
        peaks, launches = self.search_staged(staged, timers, dm_ranges)
        t2 = time.perf_counter()
        tobs = self.nsamples * self.tsamp if observation_seconds is None else observation_seconds
        if self.device_candidates:
            launches += len(peaks) + 9      # expansion per batch, keys, splits, gather (plus the sorts and scans)
            cands, npeaks = self._device_candidates(peaks, tobs)
            peaks = np.zeros(0, _lib.PEAK_DTYPE)
        else:
            peaks = core.sort_peaks(peaks)
            npeaks = len(peaks)
            cands = core.select_candidates(peaks, tobs, self.frequency_cluster_radius, self.dm_cluster_radius)
        # the step after candidate selection in the reference's drivers
        # (cuda_dm_search_benchmark.cpp:287-292)
        ranked, rel = core.flag_harmonics(cands, tobs, self.frequency_low_mhz, self.frequency_high_mhz,
                                          self.harmonic_options)
        unique = core.remove_harmonics(ranked, rel)
        t3 = time.perf_counter()
        prof = expo = None
        if len(cands):
            prof, expo = self.fold_candidate(staged, int(cands[0]["dm_index"]), float(cands[0]["period"]))
            launches += 3
        t4 = time.perf_counter()
        t.update(stage=t1 - t0, search=t2 - t1, candidates=t3 - t2, fold=t4 - t3, total=t4 - t0)
        return SearchResult(peaks=peaks, candidates=cands, fold_profile=prof, fold_exposure=expo, nout=self.nout,
                            ndm=self.ndm, timings=t, gpu_launches=launches + 1, ranked=ranked, harmonics=rel,
                            unique_candidates=unique, peak_count=npeaks)


def from_config(cfg, **overrides) -> DmSearch:
    """A DmSearch for a configs.SearchConfig workload."""
    obs = cfg.obs
    kw = dict(frequency_mhz=obs.frequencies, nsamples=obs.nsamples, tsamp=obs.tsamp, dm_low=cfg.dm_low,
              dm_step=cfg.dm_step, ndm=cfg.ndm, period_min=cfg.period_min, period_max=cfg.period_max,
              bins_min=cfg.bins_min, bins_max=cfg.bins_max, duty_cycle_max=cfg.duty_cycle_max,
              width_trials=cfg.width_trials, window_seconds=cfg.window_seconds, min_points=cfg.min_points,
              snr_threshold=cfg.snr_threshold, nbits=obs.nbits, algorithm=cfg.dedispersion,
              subband_channels=cfg.subband_channels, ndm_per_nominal=cfg.ndm_per_nominal,
              frequency_cluster_radius=cfg.frequency_cluster_radius, dm_cluster_radius=cfg.dm_cluster_radius,
              fold_nbin=cfg.fold_nbin, device_candidates=cfg.device_candidates)
    kw.update(overrides)
    return DmSearch(**kw)
