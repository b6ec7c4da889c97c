"""Small single-stage cases of the survey-size workload, for timing and for
profiler captures of one kernel family at a time.

    python -m gaffa_b200.profile_case ffa [--series 8]
        FFA search (all task classes) over `series` unit-variance noise series
        of the survey-size length (8,357,464 samples, periods 0.1-10 s,
        duty cycle <= 0.1), two searches.
    python -m gaffa_b200.profile_case dedisp [--nsamples-log2 18] [--ndm 256] [--dm-begin 1536]
        Brute-force dedispersion of the survey-size band (4096 channels,
        1100-1700 MHz, DMs 0-1000 in 2048 steps) on a shorter observation,
        `ndm` DMs from `dm_begin`, three runs.

Each prints one line per run with the CUDA-event time.
"""
from __future__ import annotations

import argparse

import torch

from . import configs, core, search

SURVEY_NOUT = 8357464  # valid output samples of the survey-size observation


def _timed(fn) -> float:
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def ffa(series: int) -> None:
    cfg = configs.survey_size()
    plan = core.make_riptide_ffa_plan(SURVEY_NOUT, cfg.obs.tsamp, cfg.period_min, cfg.period_max,
                                      bins_min=cfg.bins_min, bins_max=cfg.bins_max,
                                      duty_cycle_max=cfg.duty_cycle_max)
    prog = core.FfaProgram(plan, max_series=series)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.randn((series, SURVEY_NOUT), device="cuda", generator=g)
    prep = prog.prepare(x, series)
    torch.cuda.synchronize()
    for _ in range(2):
        ms = _timed(lambda: prog.search_async(prep, series, cfg.snr_threshold))
        print(f"ffa search ms {ms:.3f} series {series} launches {prog.kernel_launches} "
              f"peaks {int(prog.counters[0])}", flush=True)


def dedisp(nsamples_log2: int, ndm: int, dm_begin: int) -> None:
    cfg = configs.survey_size(nsamples=1 << nsamples_log2)
    raw = core.synth_generate(cfg.obs)
    ds = search.from_config(cfg, dm_batch=ndm)
    staged = ds.stage(raw)
    torch.cuda.synchronize()
    for _ in range(3):
        ms = _timed(lambda: ds.dedisp.run(staged, dm_begin, ndm, out=ds._series, out_stride=ds.out_stride))
        adds = ndm * cfg.obs.nchans * ds.nout
        print(f"dedisp ms {ms:.3f} adds/s {adds / (ms / 1e3):.3e} nout {ds.nout}", flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="case", required=True)
    f = sub.add_parser("ffa")
    f.add_argument("--series", type=int, default=8)
    d = sub.add_parser("dedisp")
    d.add_argument("--nsamples-log2", type=int, default=18)
    d.add_argument("--ndm", type=int, default=256)
    d.add_argument("--dm-begin", type=int, default=1536)
    a = ap.parse_args()
    if a.case == "ffa":
        ffa(a.series)
    else:
        dedisp(a.nsamples_log2, a.ndm, a.dm_begin)


if __name__ == "__main__":
    main()
