"""Regenerate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference sources are available, after
``make -C oracle all`` has built ``oracle/_ref/libgaffa_ref.so`` (the
reference's CPU sources compiled where they lie).  Every output below comes
from the reference's own functions through ``oracle/ref_shim.cpp``:

    python tests/golden/make_golden.py [--skip-plain]

Writes
  ref_small.npz            small seeded cases for every hot-path function
  ref_harmonic.npz         seeded candidate lists through flag_harmonics_cpu
  ref_spectrum.npz         aligned single-DM spectra (dedisperse_spectrum_cpu)
  ref_filterbank.npz       read_filterbank of the reference's tests/data/basetest.fil:
                           header fields, frequencies, sample digest, first rows
  ref_plain_end_to_end.npz the full plain end-to-end workload (256 ch, 2^18
                           samples, 512 DMs): digests of the dedispersed block
                           and of all raw peaks, the candidate list and the
                           folded profile of the top candidate
"""
from __future__ import annotations

import argparse
import os
import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gaffa_b200 import configs, synth  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small_cases(ref: Oracle) -> dict:
    out = {}
    rng = np.random.default_rng(1234)
    # multi-DM and subband dedispersion, full and partial channel ranges
    obs = synth.Observation(nchans=64, nsamples=6000, tsamp=1e-3, f_low=1200.0,
                            f_high=1500.0, seed=7,
                            pulsars=[synth.Pulsar(0.25, 30.0, 0.05, 40.0)])
    data = synth.generate(obs)
    f = obs.frequencies
    out["dd_data"] = data
    out["dd_freq"] = f
    out["dd_multi"] = ref.dedisperse_multi_dm(data, f, 0.0, 2.5, 24, f.max(), obs.tsamp)
    out["dd_multi_sub"] = ref.dedisperse_multi_dm(data, f, 3.0, 1.25, 17, f.max(),
                                                  obs.tsamp, 5, 61)
    out["dd_subband"] = ref.dedisperse_subband(data, f, 0.0, 2.5, 24, f.max(),
                                               obs.tsamp, 16, 4)
    out["dd_subband_ragged"] = ref.dedisperse_subband(data, f, 1.0, 1.5, 23, f.max(),
                                                      obs.tsamp, 12, 5, 3, 64)
    # 2-bit input: the reference path on the unpacked levels
    obs2 = synth.Observation(nchans=64, nsamples=5000, tsamp=1e-3, f_low=300.0,
                             f_high=400.0, nbits=2, seed=11,
                             pulsars=[synth.Pulsar(0.3, 20.0, 0.05, 12.0)])
    lv = synth.generate(obs2)
    out["dd2_packed"] = synth.pack_2bit(lv)
    out["dd2_freq"] = obs2.frequencies
    out["dd2_multi"] = ref.dedisperse_multi_dm(lv, obs2.frequencies, 0.0, 0.5, 20,
                                               obs2.frequencies.max(), obs2.tsamp)
    out["dd2_subband"] = ref.dedisperse_subband(lv, obs2.frequencies, 0.0, 0.5, 20,
                                                obs2.frequencies.max(), obs2.tsamp, 16, 8)
    # preprocessing: scrunched (window 1 s at 1 ms -> 1001 samples, scrunch 9)
    # and exact (window 51 < min_points) running-median paths
    x = (rng.normal(size=20000) * 30 + 500 + 40 * np.sin(np.arange(20000) / 900.0))
    x = np.round(x).astype(np.float32)
    out["pp_in"] = x
    out["pp_scrunched"] = ref.preprocess(x, 1e-3, window_seconds=1.0, min_points=101)
    out["pp_exact"] = ref.preprocess(x, 1e-3, window_seconds=0.051, min_points=101)
    out["pp_scrunched_raw"] = ref.preprocess(x, 1e-3, window_seconds=1.0, min_points=101,
                                             normalise=False)
    # downsampling and noise model
    y = rng.normal(size=4099).astype(np.float32)
    out["ds_in"] = y
    for name, fct in (("ds_a", 2.0), ("ds_b", 8.6805555), ("ds_c", 17.3611111),
                      ("ds_d", 3.5)):
        out[name] = ref.downsample(y, fct)
        out[name + "_factor"] = np.float64(fct)
        out[name + "_var"] = np.float64(ref.downsampled_variance(len(y), fct))
    # FFA transforms of odd, even and tiny shapes
    for rows, bins in ((37, 19), (64, 180), (5, 4), (2, 7), (1, 9), (129, 200)):
        z = rng.normal(size=rows * bins).astype(np.float32)
        out[f"ffa_in_{rows}x{bins}"] = z
        out[f"ffa_out_{rows}x{bins}"] = ref.ffa_transform(z, bins)
    # FFA plans
    for key, (n, ts, pmin, pmax, kw) in {
        "plan_a": (29527, 64e-6, 0.2, 2.0, {}),
        "plan_b": (258903, 64e-6, 0.2, 2.0, {}),
        "plan_c": (8357464, 64e-6, 0.1, 10.0, {"duty_cycle_max": 0.1}),
        "plan_d": (64, 0.25, 1.0, 4.0, dict(bins_min=4, bins_max=5, min_periods=2,
                                            duty_cycle_max=0.5, max_tasks=1000)),
    }.items():
        tasks, widths = ref.make_plan(n, ts, pmin, pmax, **kw)
        out[key + "_tasks"] = tasks
        out[key + "_widths"] = widths
    # single-series search over a normalised series with a periodic pulse
    n = 40000
    s = rng.normal(size=n).astype(np.float32)
    ph = (np.arange(n) * 1e-3 / 0.377) % 1.0
    s += (3.0 * np.exp(-0.5 * ((ph - 0.5) / 0.01) ** 2)).astype(np.float32)
    s = ref.preprocess(s, 1e-3, window_seconds=1.0)
    tasks, widths = ref.make_plan(n, 1e-3, 0.2, 1.5, bins_min=40, bins_max=64)
    out["search_in"] = s
    out["search_tasks"] = tasks
    out["search_widths"] = widths
    out["search_peaks"] = ref.ffa_search(s, tasks, widths, snr_threshold=3.0)
    out["search_peaks_w"] = ref.ffa_search(s, tasks, np.array([1, 2, 5, 11], np.uint64),
                                           snr_threshold=2.0)
    # candidates over a synthetic multi-DM block (uint32 sums)
    blk = out["dd_multi"]
    peaks = ref.find_dm_peaks(blk, np.arange(24) * 2.5, 1e-3,
                              dict(period_min=0.1, period_max=1.0, bins_min=40,
                                   bins_max=64),
                              dict(window_seconds=0.5, min_points=11), 5.0)
    out["dm_peaks"] = peaks
    out["cands_default"] = ref.select_candidates(peaks, blk.shape[1] * 1e-3)
    out["cands_r3_w"] = ref.select_candidates(peaks, blk.shape[1] * 1e-3,
                                              frequency_cluster_radius=0.5,
                                              dm_cluster_radius=3,
                                              cluster_across_widths=False,
                                              max_candidates=5)
    # folding
    out["fold_in_u32"] = blk[3]
    prof, expo = ref.fold(blk[3], 0.25, 1e-3, 32)
    out["fold_u32_profile"], out["fold_u32_exposure"] = prof, expo
    prof, expo = ref.fold(out["pp_scrunched"], 0.1234, 1e-3, 50, start_sample=17)
    out["fold_f32_profile"], out["fold_f32_exposure"] = prof, expo
    return out


def plain_end_to_end(ref: Oracle) -> dict:
    cfg = configs.plain_end_to_end()
    obs = cfg.obs
    t0 = time.time()
    data = synth.generate(obs)
    f = obs.frequencies
    dd = ref.dedisperse_multi_dm(data, f, cfg.dm_low, cfg.dm_step, cfg.ndm,
                                 obs.ref_frequency, obs.tsamp)
    t1 = time.time()
    peaks = ref.find_dm_peaks(dd, cfg.dms, obs.tsamp, cfg.plan_options(),
                              cfg.preprocess_options(), cfg.snr_threshold,
                              widths=np.array(cfg.width_trials, np.uint64))
    t2 = time.time()
    # observation length as the reference's pipeline driver passes it
    # (cuda_dm_search_benchmark.cpp: header.tsamp * header.nsamples)
    tobs = obs.nsamples * obs.tsamp
    cands = ref.select_candidates(peaks, tobs, cfg.frequency_cluster_radius,
                                  cfg.dm_cluster_radius)
    top = cands[0]
    prof, expo = ref.fold(dd[int(top["dm_index"])], float(top["period"]), obs.tsamp,
                          cfg.fold_nbin)
    print(f"plain_end_to_end: dedisperse {t1 - t0:.1f}s search {t2 - t1:.1f}s "
          f"peaks {len(peaks)} candidates {len(cands)}")
    return {
        "input_digest": np.array(digest(data)),
        "nout": np.int64(dd.shape[1]),
        "dedispersed_digest": np.array(digest(dd)),
        "dedispersed_rows": dd[[0, 1, 255, 511]],
        "npeaks": np.int64(len(peaks)),
        "peaks_digest": np.array(digest(peaks)),
        "peaks_top": peaks[:4096],
        "candidates": cands,
        "fold_profile": prof,
        "fold_exposure": expo,
    }


def harmonic_candidates(rng: np.random.Generator, n: int) -> np.ndarray:
    """Candidate lists with harmonic families: parents at random frequencies,
    children at n/d multiples (small frequency jitter), nearby DMs, and
    unrelated candidates."""
    from oracle.oracle import CAND_DTYPE
    c = np.zeros(n, CAND_DTYPE)
    nparent = max(1, n // 4)
    pf = rng.uniform(0.1, 10.0, nparent)
    pdm = rng.uniform(0.0, 500.0, nparent)
    for i in range(n):
        if i < nparent:
            f, dm = pf[i], pdm[i]
        elif rng.random() < 0.7:
            j = rng.integers(nparent)
            num, den = rng.integers(1, 9), rng.integers(1, 6)
            f = pf[j] * num / den * (1.0 + rng.normal(0, 2e-4))
            dm = pdm[j] + rng.normal(0, 2.0)
        else:
            f, dm = rng.uniform(0.1, 10.0), rng.uniform(0.0, 500.0)
        duty = rng.choice([0.01, 0.02, 0.05, 0.1])
        c[i]["frequency"] = f
        c[i]["period"] = 1.0 / f
        c[i]["dm"] = max(dm, 0.0)
        c[i]["dm_index"] = int(max(dm, 0.0) * 2)
        c[i]["duty_cycle"] = duty
        c[i]["width"] = max(1, int(round(duty * 200)))
        c[i]["snr"] = np.float32(rng.uniform(6.0, 40.0))
        c[i]["peak_count"] = rng.integers(1, 50)
        c[i]["dm_index_min"] = c[i]["dm_index"]
        c[i]["dm_index_max"] = c[i]["dm_index"]
        c[i]["frequency_min"] = f
        c[i]["frequency_max"] = f
    return c


def harmonic_cases(ref: Oracle) -> dict:
    out = {}
    rng = np.random.default_rng(4321)
    options = [dict(), dict(max_harmonic=8, denominator_max=3), dict(frequency_tolerance_bins=3.0,
               phase_distance_max=2.0, dm_distance_max=10.0), dict(use_snr_consistency=True, snr_distance_max=5.0)]
    for k, opts in enumerate(options):
        cands = harmonic_candidates(rng, 60 + 20 * k)
        ctx = (rng.uniform(50.0, 600.0), 1100.0, 1700.0)
        srt, rel = ref.flag_harmonics(cands, *ctx, **opts)
        out[f"h{k}_in"] = cands
        out[f"h{k}_ctx"] = np.array(ctx)
        out[f"h{k}_sorted"] = srt
        out[f"h{k}_rel"] = rel
        out[f"h{k}_kept"] = ref.remove_harmonics(srt, rel, 10)
    # the plain end-to-end candidate list, as the pipeline flags it
    plain = OUT / "ref_plain_end_to_end.npz"
    if plain.exists():
        cfg = configs.plain_end_to_end()
        f = cfg.obs.frequencies
        ctx = (cfg.obs.nsamples * cfg.obs.tsamp, float(f.min()), float(f.max()))
        srt, rel = ref.flag_harmonics(np.load(plain)["candidates"], *ctx)
        out["plain_ctx"] = np.array(ctx)
        out["plain_sorted"] = srt
        out["plain_rel"] = rel
    return out


def spectrum_cases(ref: Oracle) -> dict:
    obs = synth.Observation(nchans=48, nsamples=3000, tsamp=1e-3, f_low=1200.0, f_high=1500.0, seed=5,
                            pulsars=[synth.Pulsar(0.2, 60.0, 0.05, 40.0)])
    data = synth.generate(obs)
    f = obs.frequencies
    out = {"sp_data": data, "sp_freq": f}
    out["sp_full"] = ref.dedisperse_spectrum(data, f, 60.0, f.max(), obs.tsamp)
    out["sp_sub"] = ref.dedisperse_spectrum(data, f, 37.5, f.max(), obs.tsamp, 5, 41)
    out["sp_zero"] = ref.dedisperse_spectrum(data, f, 0.0, f.max(), obs.tsamp)
    # fold of the aligned spectrum at the pulsar's period
    for tag, kw in (("fold", dict(nbin=32, tsubint=0.5)), ("fold_ch", dict(nbin=24, tsubint=0.7, output_channels=12))):
        r = ref.fold_dedispersed_spectrum(out["sp_full"], 0.2, obs.tsamp, **kw)
        for k, v in r.items():
            out[f"{tag}_{k}"] = v
    return out


def filterbank_cases(ref: Oracle) -> dict:
    path = Path(ref_dir()) / "tests" / "data" / "basetest.fil"
    out = {}
    for tag, preserve in (("asc", False), ("file", True)):
        h, f, data = ref.read_filterbank(path, preserve)
        for k, v in h.items():
            out[f"{tag}_h_{k}"] = np.array(v)
        out[f"{tag}_freq"] = f
        out[f"{tag}_digest"] = np.array(digest(data))
        out[f"{tag}_head"] = data[: 64 * 1024]
    return out


def ref_dir() -> str:
    """The gaffa checkout the fixtures come from (GAFFA_REFERENCE_DIR)."""
    path = os.environ.get("GAFFA_REFERENCE_DIR")
    if not path:
        raise SystemExit("set GAFFA_REFERENCE_DIR to the gaffa checkout")
    return path


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-small", action="store_true")
    args = ap.parse_args()
    ref = Oracle("reference")
    np.savez_compressed(OUT / "ref_harmonic.npz", **harmonic_cases(ref))
    np.savez_compressed(OUT / "ref_spectrum.npz", **spectrum_cases(ref))
    np.savez_compressed(OUT / "ref_filterbank.npz", **filterbank_cases(ref))
    if not args.skip_small:
        np.savez_compressed(OUT / "ref_small.npz", **small_cases(ref))
    if not args.skip_plain:
        np.savez_compressed(OUT / "ref_plain_end_to_end.npz", **plain_end_to_end(ref))


if __name__ == "__main__":
    main()
