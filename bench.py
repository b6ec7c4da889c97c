#!/usr/bin/env python3
"""Benchmark: DM-trial·samples/s of the full pulsar search on B200.

One step = the whole search of one observation: stage the filterbank,
dedisperse every DM trial, detrend + normalise, downsample per octave, FFA +
boxcar S/N over every task, expand and sort peaks, select candidates and fold
the best one.  `value` times steps whose filterbank is already resident in
HBM; `e2e` times the same search through the public pipeline API from a
pinned host filterbank (host->device copy inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gaffa|reference]

The same line carries measurements of the other workloads on rank 0: the
learned proposal, two batched uneven workloads, the wide-range subband
configuration at its size (`--no-proposal`, `--no-batched`,
`--no-wide-subband` skip them), and, with `--batched-configured`, the
batched workload at its configured laws (64 observations, ~20 minutes).

Multi-GPU runs (torchrun) are replicas: every rank searches its own
observation (weak scaling); time is the max over ranks.  `--impl reference`
times the reference's own CPU implementation (compiled from its sources,
oracle/_ref) on a bounded sample of DM trials of the same workload, on all
host cores of rank 0.
"""
from __future__ import annotations

import argparse
import functools
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DM-trial·samples/s searched"
UNIT = "DM-trial·samples/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) one FFA search moves per DM-trial series, from an
# ncu capture of the survey-size FFA plan (recorded with its command)
FFA_TRAFFIC_FILE = ROOT / "profiles" / "ffa_search_kernel_survey_size.json"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gaffa", "reference"], default="gaffa")
    ap.add_argument("--workload", default="survey_size")
    ap.add_argument("--ndm", type=int, default=None, help="override the DM-trial count (testing)")
    ap.add_argument("--nsamples-log2", type=int, default=None, help="override the length (testing)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-dms", type=int, default=8,
                    help="DM trials in the CPU baseline sample (at least 5, the reference's parallel DM path)")
    ap.add_argument("--no-proposal", action="store_true", help="skip the learned-proposal measurement")
    ap.add_argument("--proposal-fraction", type=float, default=None,
                    help="fraction of DM windows searched (default: the shipped model's)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched uneven-workload measurement")
    ap.add_argument("--batched-observations", type=int, default=12)
    ap.add_argument("--batched-configured", action="store_true",
                    help="also run the batched workload at its configured laws (64 observations, ~15 minutes)")
    ap.add_argument("--no-wide-subband", action="store_true",
                    help="skip the wide-range subband measurement at its configured size")
    return ap.parse_args()


def workload(args, rank: int = 0):
    from gaffa_b200 import configs
    kw = {}
    if args.ndm:
        kw["ndm"] = args.ndm
    if args.nsamples_log2:
        kw["nsamples"] = 1 << args.nsamples_log2
    return configs.CONFIGS[args.workload](seed=rank, **kw)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.lines: list[str] = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def ffa_traffic_per_series(workload: str):
    """traffic_bytes_per_series of the recorded FFA capture (survey size only)."""
    if workload != "survey_size":
        return None
    try:
        return float(json.loads(FFA_TRAFFIC_FILE.read_text())["traffic_bytes_per_series"])
    except (OSError, KeyError, ValueError):
        return None


def measured_hbm_gbs():
    try:
        return float(json.loads(PEAKS_FILE.read_text())["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# Per-unit algorithmic bytes (one unit = one DM-trial x one output sample).
def algorithmic_bytes(stage: str, cfg, ds, units: int) -> float:
    obs = cfg.obs
    if stage == "dedisperse":
        # input read once + uint32 output written
        in_bytes = obs.nsamples * obs.nchans * (1 if obs.nbits == 8 else 0.25)
        per_unit = 4.0 + in_bytes / (cfg.ndm * ds.nout)
        if cfg.dedispersion == "subband":
            # plus the uint8 stage-1 intermediate, written once and read once
            n_nom = -(-cfg.ndm // cfg.ndm_per_nominal)
            inter = float(n_nom) * (obs.nchans // cfg.subband_channels) * obs.nsamples
            per_unit += 2.0 * inter / (cfg.ndm * ds.nout)
        return units * per_unit
    if stage == "preprocess":
        return units * 8.0                    # uint32 in, float out, in place
    if stage == "prepare":
        return units * 4.0 + units / ds.nout * ds.ffa.prepared_floats * 4.0
    if stage == "ffa":
        # prepared block read once per task (rows*bins per task) per series
        per_series = float(sum(int(t["rows"]) * int(t["bins"]) for t in ds.plan.tasks)) * 4.0
        return units / ds.nout * per_series
    return 0.0


def set_cpu_threads() -> None:
    """OpenMP settings for the CPU legs (before any OpenMP runtime starts):
    one thread per physical core, threads bound close, one place per core
    (as the reference's own benchmark recipes run it)."""
    os.environ.setdefault("OMP_NUM_THREADS", str(host_cpu()["physical_cores"]))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")


@functools.lru_cache(maxsize=None)
def host_cpu() -> dict:
    """The host's CPU model and core counts (the cores this process may use),
    read once before any OpenMP runtime binds this thread to one core."""
    logical = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil
        physical = psutil.cpu_count(logical=False) or logical
    except ImportError:
        physical = logical
    physical = max(1, min(physical, logical))
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "physical_cores": physical, "logical_cpus": logical}


class ReferenceCpuPath:
    """The reference's own CPU implementation of the path (oracle/_ref: its
    sources compiled where they lie; else the C restatement) on a contiguous
    sample of DM trials at full length: dedisperse_multi_dm_cpu (or
    dedisperse_subband_cpu on the unpacked 2-bit levels), find_dm_peaks_cpu
    (convert, detrend, normalise, FFA, S/N), select_candidates_cpu and
    fold_time_series_cpu of the best candidate -- the chain of
    dm_search.cpp:142-199 and candidate.cpp:35-212."""

    def __init__(self, cfg, data: np.ndarray):
        from oracle.oracle import Oracle
        self.kind = "reference" if Oracle.available("reference") else "port"
        self.ref = Oracle(self.kind)
        self.cfg = cfg
        obs = cfg.obs
        if obs.nbits == 2:
            from gaffa_b200 import synth  # numpy only
            data = synth.unpack_2bit(data, obs.nchans)   # the reference has no packed-input path
        self.data = data
        self.nout = self.ref.output_nsamples(obs.frequencies, obs.nsamples, cfg.dm_low, cfg.dm_step, cfg.ndm,
                                             obs.ref_frequency, obs.tsamp)
        self.widths = None if cfg.width_trials is None else np.array(cfg.width_trials, np.uint64)

    def sample_size(self, minimum: int) -> int:
        """DM trials per step: at least `minimum`, and for subband dedispersion
        whole nominal-DM groups, so stage 1 is amortised as in a full run."""
        cfg = self.cfg
        n = minimum
        if cfg.dedispersion == "subband":
            g = cfg.ndm_per_nominal
            n = max(g, (n + g - 1) // g * g)
        return min(n, cfg.ndm)

    def first_dm(self, nsel: int) -> int:
        """A contiguous sample in the middle of the DM range (aligned to the
        nominal-DM groups for subband dedispersion)."""
        cfg = self.cfg
        b0 = (cfg.ndm - nsel) // 2
        if cfg.dedispersion == "subband":
            b0 -= b0 % cfg.ndm_per_nominal
        return max(0, b0)

    def step(self, nsel: int) -> float:
        cfg, obs, ref = self.cfg, self.cfg.obs, self.ref
        b0 = self.first_dm(nsel)
        dm0 = cfg.dm_low + b0 * cfg.dm_step
        t0 = time.perf_counter()
        if cfg.dedispersion == "subband":
            blk = ref.dedisperse_subband(self.data, obs.frequencies, dm0, cfg.dm_step, nsel, obs.ref_frequency,
                                         obs.tsamp, subband_channels=cfg.subband_channels,
                                         ndm_per_nominal=cfg.ndm_per_nominal)
        else:
            blk = ref.dedisperse_multi_dm(self.data, obs.frequencies, dm0, cfg.dm_step, nsel, obs.ref_frequency,
                                          obs.tsamp)
        blk = np.ascontiguousarray(blk[:, : self.nout])
        peaks = ref.find_dm_peaks(blk, cfg.dms[b0:b0 + nsel], obs.tsamp, cfg.plan_options(),
                                  cfg.preprocess_options(), cfg.snr_threshold, widths=self.widths)
        cands = ref.select_candidates(peaks, obs.nsamples * obs.tsamp)
        if len(cands):
            # DmPeak::dm_index indexes the rows of the searched block
            ref.fold(blk[int(cands[0]["dm_index"])], float(cands[0]["period"]), obs.tsamp, cfg.fold_nbin)
        return time.perf_counter() - t0

    def describe(self, nsel: int, seconds: float) -> str:
        cfg = self.cfg
        b0 = self.first_dm(nsel)
        dd = "dedisperse_subband_cpu" if cfg.dedispersion == "subband" else "dedisperse_multi_dm_cpu"
        return (f"DM trials {b0}-{b0 + nsel - 1} of {cfg.ndm} (contiguous), full length ({self.nout} samples): "
                f"{dd} + find_dm_peaks_cpu + select_candidates_cpu + fold_time_series_cpu, {seconds:.1f} s; "
                f"{os.environ.get('OMP_NUM_THREADS')} OpenMP threads, OMP_PROC_BIND="
                f"{os.environ.get('OMP_PROC_BIND')}, OMP_PLACES={os.environ.get('OMP_PLACES')}")


# find_dm_peaks_cpu runs its DM loop in parallel only for more than 4 trials
# (dm_search.cpp:160), so every reference sample holds at least 5
REFERENCE_MIN_DMS = 5


def run_reference(args, rank: int, world: int) -> None:
    """Reference CPU implementation (oracle/_ref, else the port) on a bounded
    DM-trial sample of the workload, with every physical host core.  The input
    is the same seeded observation, generated on the host cores by the
    checkers' generator (oracle/synth_oracle.c), so this arm never loads the
    CUDA library."""
    if rank != 0:
        return
    from oracle import oracle
    cfg = workload(args)
    obs = cfg.obs
    cpu = host_cpu()
    t0 = time.perf_counter()
    data = oracle.synth_generate(obs)
    gen_s = time.perf_counter() - t0
    path = ReferenceCpuPath(cfg, data)
    nsel = path.sample_size(REFERENCE_MIN_DMS)
    # the CPU path has no device state or compilation to warm: one untimed
    # step faults in the pages, then K timed steps
    path.step(nsel)
    times = [path.step(nsel) for _ in range(args.steps)]
    sec = sum(times) / len(times)
    value = nsel * path.nout / sec
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": 1, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": {"workload": cfg.name, "nchans": obs.nchans, "nsamples": obs.nsamples, "nbits": obs.nbits,
                   "ndm": cfg.ndm, "nout": path.nout, "dedispersion": cfg.dedispersion},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
                         "kind": path.kind, "cpu": cpu,
                         "sample": path.describe(nsel, sec) + f"; input generated in {gen_s:.1f} s (untimed)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def proposal_measurement(cfg, ds, raw, exhaustive, fraction):
    """The learned-proposal path on the same observation: the coarse search,
    the network's window scores, then the full-resolution search of the top
    fraction of DM windows.  Throughput counts every DM trial of the
    observation (the ones the proposal rules out included); recall is over
    the injections the exhaustive search itself detected."""
    import torch
    from gaffa_b200 import proposal
    obs = cfg.obs
    dev = ds.device.index or 0
    net = proposal.ProposalNet(device_id=dev)
    meta = net.load_default()
    frac = fraction if fraction is not None else meta["fraction"]
    dm_max = cfg.dm_low + (cfg.ndm - 1) * cfg.dm_step
    cf = proposal.CoarseFeatures(obs.frequencies, obs.nsamples, obs.tsamp, dm_max, device_id=dev)

    def run_once():
        feats = cf(raw)
        scores = net.forward(feats)
        windows = proposal.select_windows(scores, frac)
        ranges = proposal.dm_ranges_for_windows(windows, cfg.ndm, cfg.dm_step, dm_max, ds.dedisp.batch_granularity)
        return feats, windows, ranges, ds.run(raw, dm_ranges=ranges)

    run_once()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    feats, windows, ranges, _ = run_once()
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    det = proposal.detected_injections(exhaustive.candidates, obs.pulsars, obs.nsamples * obs.tsamp,
                                       cfg.snr_threshold, proposal.band_delay_per_dm(obs.frequencies))
    found, total = proposal.injection_recall(det, windows, dm_max)
    hfound, _ = proposal.injection_recall(det, proposal.select_windows(proposal.baseline_scores(feats), frac),
                                          dm_max)
    return {"value": cfg.ndm * ds.nout / sec, "unit": UNIT, "ms_per_step": sec * 1e3, "window_fraction": frac,
            "dm_trials_searched": int(sum(e - b for b, e in ranges)), "injections_detected_exhaustive": total,
            "injections_recalled": found, "recall": (found / total) if total else None,
            "heuristic_recalled_same_budget": hfound, "model": meta.get("trained_on", ""),
            "model_val_recall_at_fraction": meta.get("val_recall_at_fraction")}


BATCHED_CASES = {
    # the batched laws at reduced lengths and DM counts
    "reduced": dict(log2_nsamples=(18.0, 20.0), ndm_range=(256, 1024)),
    # many small observations, where launches and host round trips dominate
    "small": dict(nchans_choices=(256, 512, 1024), log2_nsamples=(16.0, 18.0), ndm_range=(64, 256)),
}


def batched_measurement(nobs: int, device_id: int, case: str = "reduced") -> dict:
    """A batched uneven workload (BATCHED_CASES: the batched laws, channels
    from {1024, 2048, 4096} or smaller, own FFA period ranges, 0-4 pulsars).
    Times one batched run (one dedispersion launch and one FFA launch per
    class per wave, replayed from captured CUDA graphs, autotuned
    dedispersion shapes) against the same observations searched one after
    another by DmSearch, both from HBM-resident filterbanks, and checks that
    the peaks and candidates agree."""
    import numpy as np
    import torch
    from gaffa_b200 import batch, configs, core, search
    cs = configs.batched_uneven(seed=0, nobs=nobs, **BATCHED_CASES[case])
    data = [core.synth_generate(c.obs, device_id=device_id) for c in cs]
    tuner = batch.Autotuner()
    t0 = time.perf_counter()
    bs = batch.BatchSearch(cs, device_id=device_id, tuner=tuner)
    first = bs.run(data)                       # tunes, builds the waves, captures the graphs
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    units = sum(c.ndm * dd.nout for c, dd in zip(cs, bs.dd))

    def timed(fn):
        torch.cuda.synchronize()
        a = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - a, out

    sec_replay, got = timed(lambda: bs.run())         # staged data resident: graph replays only
    split = {}
    sec_b, _ = timed(lambda: bs.run(data, timers=split))  # with the staging of every filterbank
    searches = [search.from_config(c, device_id=device_id) for c in cs]
    for s, x in zip(searches, data):
        s.run(x)                                     # warm-up
    sec_s, want = timed(lambda: [s.run(x) for s, x in zip(searches, data)])
    same = all(np.array_equal(a.peaks, b.peaks) and np.array_equal(a.candidates, b.candidates)
               for a, b in zip(got, want)) and all(np.array_equal(a.peaks, b.peaks) for a, b in zip(first, want))
    waves = len(bs.waves)
    launches = bs.kernel_launches_per_run
    del bs, searches, data
    torch.cuda.empty_cache()
    return {"value": units / sec_b, "unit": UNIT, "observations": nobs, "dm_trial_samples": units, "waves": waves,
            "kernel_launches_per_run": launches, "seconds": sec_b, "seconds_staged_data": sec_replay,
            "sequential_value": units / sec_s, "sequential_seconds": sec_s, "speedup_vs_sequential": sec_s / sec_b,
            "identical_to_sequential": bool(same), "setup_seconds": setup,
            "split_seconds": {k: round(v, 4) for k, v in split.items()},
            "tuned_dedispersion_shapes": tuner.cache, "case": case, "laws": BATCHED_CASES[case]}


def batched_configured_measurement(device_id: int, nobs: int = 64, memory_fraction: float = 0.3) -> dict:
    """The batched uneven workload at its configured laws: 64 observations,
    channels from {1024, 2048, 4096}, lengths log-uniform over 2^20-2^23,
    256-4096 DM trials, own FFA period ranges, 0-4 pulsars each (631 GB of
    raw input in all).  The observations are searched in consecutive
    sub-batches whose filterbanks and staging buffers fit memory_fraction of
    the free HBM; each sub-batch is generated on the device, set up (launch
    shapes tuned, waves captured as CUDA graphs) outside the timing, then
    searched once by BatchSearch from its device filterbanks and once by
    DmSearch one observation after another.  Reports both throughputs, the
    speed-up, kernel launches per wave and whether every result is identical."""
    import torch
    from gaffa_b200 import batch, configs, core, search
    cs = configs.batched_uneven(seed=0, nobs=nobs)
    free = torch.cuda.mem_get_info(device_id)[0]
    budget = int(free * memory_fraction)
    groups, cur, used = [], [], 0
    for c in cs:
        need = 2 * c.obs.nchans * c.obs.nsamples
        if cur and used + need > budget:
            groups.append(cur)
            cur, used = [], 0
        cur.append(c)
        used += need
    if cur:
        groups.append(cur)
    tuner = batch.Autotuner()
    t_batched = t_seq = 0.0
    units = 0
    same = True
    launches, waves = [], 0

    def timed(fn):
        torch.cuda.synchronize()
        a = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - a, out

    t_first = 0.0
    for gi, sub in enumerate(groups):
        data = [core.synth_generate(c.obs, device_id=device_id) for c in sub]
        bs = batch.BatchSearch(sub, device_id=device_id, tuner=tuner)
        dt, _ = timed(lambda: bs.run(data))            # tunes shapes, builds and captures the waves
        t_first += dt
        dt, got = timed(lambda: bs.run(data))
        t_batched += dt
        units += sum(c.ndm * dd.nout for c, dd in zip(sub, bs.dd))
        launches.append(bs.kernel_launches_per_run)
        waves += len(bs.waves)
        del bs
        torch.cuda.empty_cache()
        for c, x, g in zip(sub, data, got):
            ds = search.from_config(c, device_id=device_id)
            dt, want = timed(lambda: ds.run(x))
            t_seq += dt
            same = same and np.array_equal(g.peaks, want.peaks) and np.array_equal(g.candidates, want.candidates)
            del ds
        del data
        torch.cuda.empty_cache()
        print(f"batched configured: sub-batch {gi + 1}/{len(groups)}, {len(sub)} observations, "
              f"batched {t_batched:.1f} s, sequential {t_seq:.1f} s, identical {same}", file=sys.stderr, flush=True)
    return {"value": units / t_batched, "unit": UNIT, "observations": nobs, "sub_batches": len(groups),
            "waves": waves, "dm_trial_samples": units, "seconds": t_batched, "first_run_seconds": t_first,
            "sequential_seconds": t_seq,
            "sequential_value": units / t_seq, "speedup_vs_sequential": t_seq / t_batched,
            "kernel_launches_per_sub_batch": launches, "identical_to_sequential": bool(same),
            "tuned_dedispersion_shapes": tuner.cache,
            "laws": "configs.batched_uneven: channels {1024, 2048, 4096}, 2^20-2^23 samples, 256-4096 DMs"}


def wide_subband_measurement(device_id: int) -> dict:
    """The wide-range subband workload at its configured size (2-bit, 4096
    channels over 300-400 MHz, 2^22 samples, 64 subbands, nominal DMs every
    20, 8192 DM trials over 0-3000, 16 pulsars, 50 Hz narrowband and 0.1 Hz
    impulse RFI): one warm-up and one timed search from an HBM-resident
    packed filterbank, with candidate selection on the device (its ~10^8 raw
    peaks never leave the GPU).  Reports DM-trial*samples/s, the stage times,
    the subband dedispersion's byte-add rate and algorithmic bytes, and the
    raw-peak and candidate counts."""
    import torch
    from gaffa_b200 import configs, core, search
    cfg = configs.wide_subband()
    obs = cfg.obs
    raw = core.synth_generate(obs, device_id=device_id)
    ds = search.from_config(cfg, device_id=device_id, peak_capacity=None)
    ds.run(raw)                                      # warm-up; sizes the peak buffer
    timers = {}
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    res = ds.run(raw, timers=timers)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b)
    stage = {k: round(sum(x.elapsed_time(y) for x, y in v), 2) for k, v in timers.items()}
    units = cfg.ndm * ds.nout
    n_nom = -(-cfg.ndm // cfg.ndm_per_nominal)
    n_sb = obs.nchans // cfg.subband_channels
    stage1_adds = float(n_nom) * obs.nchans * obs.nsamples
    stage2_adds = float(cfg.ndm) * n_sb * ds.nout
    # packed input read, uint8 intermediate written and read, uint32 output written
    inter = float(n_nom) * n_sb * obs.nsamples
    alg = obs.nchans * obs.nsamples / 4 + 2 * inter + 4.0 * units
    dd_s = stage.get("dedisperse", 0.0) / 1e3
    out = {"value": units / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "nout": ds.nout, "ndm": cfg.ndm,
           "dm_batch": ds.dm_batch, "stage_ms": stage, "raw_peaks": res.peak_count,
           "candidates": len(res.candidates), "candidate_selection": "device",
           "dedisperse": {"stage1_adds": stage1_adds, "stage2_adds": stage2_adds,
                          "adds_per_s": (stage1_adds + stage2_adds) / dd_s if dd_s else None,
                          "algorithmic_bytes": alg, "achieved_gbs": alg / dd_s / 1e9 if dd_s else None},
           "config": {"workload": cfg.name, "nchans": obs.nchans, "nsamples": obs.nsamples, "nbits": obs.nbits,
                      "subbands": n_sb, "ndm_per_nominal": cfg.ndm_per_nominal}}
    del ds, raw
    torch.cuda.empty_cache()
    return out


def cpu_baseline(cfg, host_input, min_dms: int) -> dict:
    """The reference CPU path on a contiguous sample of at least `min_dms` DM
    trials of the same observation (ReferenceCpuPath), timed once."""
    path = ReferenceCpuPath(cfg, host_input)
    nsel = path.sample_size(min_dms)
    dt = path.step(nsel)
    return {"value": nsel * path.nout / dt, "unit": UNIT, "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": path.kind, "cpu": host_cpu(), "sample": path.describe(nsel, dt)}


def main():
    args = parse_args()
    set_cpu_threads()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return

    from gaffa_b200 import core, search
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    batched = batched_small = wide = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched = batched_measurement(args.batched_observations, local, "reduced")
        batched_small = batched_measurement(64, local, "small")
    if rank == 0 and world == 1 and not args.no_wide_subband and args.workload != "wide_subband":
        wide = wide_subband_measurement(local)
    batched_configured = None
    if rank == 0 and world == 1 and args.batched_configured:
        batched_configured = batched_configured_measurement(local)
    cfg = workload(args, rank)
    obs = cfg.obs
    raw = core.synth_generate(obs, device_id=local)          # device-resident filterbank
    ds = search.from_config(cfg, device_id=local)
    timers = {}

    def step(src):
        return ds.run(src, timers=timers)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(src, k):
        timers.clear()
        barrier()
        torch.cuda.synchronize(device)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        res = None
        for _ in range(k):
            res = step(src)
        b.record()
        torch.cuda.synchronize(device)
        barrier()
        ms = a.elapsed_time(b) / k
        if dist is not None:
            t = torch.tensor([ms], device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, res

    for _ in range(args.warmup):
        step(raw)
    with ClockSampler(local) as clk:
        ms, res = timed(raw, args.steps)
    stage_ms = {k: [s.elapsed_time(e) for s, e in v] for k, v in timers.items()}
    clocks = clk.summary()
    units = cfg.ndm * ds.nout
    value = units * world / (ms / 1e3)

    # roofline of the dominant stage
    peak, peak_kind = measured_hbm_gbs()
    totals = {k: sum(v) for k, v in stage_ms.items() if v}
    dominant = max(totals, key=totals.get)
    per_launch_ms = totals[dominant] / len(stage_ms[dominant])
    launches_per_step = len(stage_ms[dominant]) / args.steps
    units_per_launch = units / launches_per_step
    alg = algorithmic_bytes(dominant, cfg, ds, units_per_launch)
    achieved = alg / (per_launch_ms / 1e3) / 1e9
    traffic = None
    series_per_launch = units_per_launch / ds.nout
    if dominant == "ffa" and ffa_traffic_per_series(cfg.name) is not None:
        traffic = ffa_traffic_per_series(cfg.name) * series_per_launch
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": dominant, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic_bytes_per_launch": alg, "launch_ms": per_launch_ms,
                "stage_ms_per_step": {k: round(v / args.steps, 3) for k, v in totals.items()}}
    # the compute roofs that bind these kernels: byte adds and FFA element-levels
    if "ffa" in totals:
        per_series = float(sum(int(t["rows"]) * int(t["bins"]) * max(1, int(t["rows"]) - 1).bit_length()
                               for t in ds.plan.tasks))
        roofline["ffa_element_levels_per_s"] = per_series * cfg.ndm / (totals["ffa"] / args.steps / 1e3)
    if "dedisperse" in totals:
        roofline["dedisperse_adds_per_s"] = float(cfg.ndm) * obs.nchans * ds.nout / (totals["dedisperse"] / args.steps / 1e3)

    e2e = None
    host = None
    if not args.no_e2e:
        host = torch.empty(raw.shape, dtype=torch.uint8, pin_memory=True)
        host.copy_(raw)
        # observations back to back from pinned host memory: each one's copies
        # overlap the previous one's search (DmSearch.run_many); the first
        # copy is inside the timed region
        ds.run_many([host])
        barrier()
        torch.cuda.synchronize(device)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        ds.run_many([host] * args.steps)
        b.record()
        torch.cuda.synchronize(device)
        barrier()
        ms_e2e = a.elapsed_time(b) / args.steps
        if dist is not None:
            t = torch.tensor([ms_e2e], device=device)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_e2e = float(t.item())
        # peak records + counters + the folded profile (float) and exposure (double)
        d2h = len(res.peaks) * 24 + 16 + ds.fold_nbin * 12
        e2e = {"value": units * world / (ms_e2e / 1e3), "unit": UNIT, "ms_per_step": ms_e2e,
               "h2d_bytes_per_step": int(raw.numel()), "d2h_bytes_per_step": d2h}

    prop = None
    if rank == 0 and world == 1 and not args.no_proposal:
        try:
            prop = proposal_measurement(cfg, ds, raw, res, args.proposal_fraction)
            prop["speedup_vs_plain"] = prop["value"] / value
        except FileNotFoundError as exc:
            prop = {"unavailable": f"no trained proposal model: {exc}"}

    baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        src = host.numpy() if host is not None else raw.cpu().numpy()
        try:
            baseline = cpu_baseline(cfg, src, max(REFERENCE_MIN_DMS, args.cpu_dms))
        except Exception as exc:  # the baseline is reported, never the target
            baseline = {"value": None, "unit": UNIT, "cores": host_cpu()["physical_cores"], "kind": "reference",
                        "sample": f"failed: {exc}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": {"workload": cfg.name, "nchans": obs.nchans, "nsamples": obs.nsamples, "nbits": obs.nbits,
                       "ndm": cfg.ndm, "nout": ds.nout, "dedispersion": cfg.dedispersion,
                       "ffa_tasks": ds.plan.task_count, "width_trials": list(ds.plan.width_trials),
                       "dm_batch": ds.dm_batch, "parallelism": f"replicas x{world}",
                       "l2": f"inputs larger than L2 ({raw.numel() / 1e9:.1f} GB filterbank)", "peaks": len(res.peaks),
                       "candidates": len(res.candidates)},
            "e2e": e2e,
            "gpu_launches": res.gpu_launches * args.steps,
            "roofline": roofline,
            "cpu_baseline": baseline,
            "proposal": prop,
            "batched": batched,
            "batched_small": batched_small,
            "wide_subband": wide,
            "batched_configured": batched_configured,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
