"""Learned DM/period proposal in front of the exhaustive search.

A coarse search runs first: the band brute-force dedispersed at 256 coarse
DMs over the search range, downsampled 8x, detrended and searched by the FFA
(every step the full search's own kernels, at a few per cent of its cost).
Its peaks give, for each of 64 DM windows, a max-S/N map over 7 period
octaves (0.1-12.8 s) x 64 log-period bins.  A small 1-D convolutional network
(csrc/proposal.cu: 32, 64, 64, 32 channels, kernel 9, then a per-bin score
pooled per octave) reads each window's map beside the zero-DM window's map
and scores the 7 octaves.

Training labels come from the exhaustive search's own candidates on seeded
synthetic injections: the windows and octaves of the candidates that match an
injected pulsar (its period or a harmonic ratio n/m, n, m <= 4, at a DM whose
smearing stays below a quarter period) are positive.  At inference the
windows are ranked by their best octave score and only the top fraction goes
to the full-resolution search (DmSearch.run(dm_ranges=...)); the exhaustive
search remains the fallback and the measure of recall.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import json
import math
from pathlib import Path

import numpy as np
import torch

from . import _lib, core, search, synth
from ._lib import check, ptr

OCTAVES = 7
BINS_PER_OCTAVE = 64
NBINS = OCTAVES * BINS_PER_OCTAVE
F_MAX = 10.0                         # Hz: period 0.1 s
F_MIN = F_MAX / 2 ** OCTAVES         # Hz: period 12.8 s
NCOARSE = 64                         # DM windows scored by the network
COARSE_DMS = 256                     # coarse DM trials of the coarse search (4 per window)
DOWNSAMPLE = 8
IN_CHANNELS = 2                      # the window's S/N map and the zero-DM window's
LAYERS = ((IN_CHANNELS, 32, 9), (32, 64, 9), (64, 64, 9), (64, 32, 9))
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "proposal_weights.npz"


def bin_edges() -> np.ndarray:
    """Log-frequency bin edges (Hz), ascending: bin j spans one 64th of an octave."""
    return (F_MIN * 2.0 ** (np.arange(NBINS + 1) / BINS_PER_OCTAVE)).astype(np.float32)


def octave_of_period(period) -> np.ndarray:
    """Octave index (0 = 6.4-12.8 s ... 6 = 0.1-0.2 s), clipped to the grid."""
    f = 1.0 / np.asarray(period, dtype=np.float64)
    j = np.floor(BINS_PER_OCTAVE * np.log2(f / F_MIN)).astype(np.int64)
    return np.clip(j // BINS_PER_OCTAVE, 0, OCTAVES - 1)


def window_of_dm(dm, dm_max: float) -> np.ndarray:
    """DM window (nearest of NCOARSE window centres over [0, dm_max])."""
    w = np.rint(np.asarray(dm, dtype=np.float64) / dm_max * (NCOARSE - 1)).astype(np.int64)
    return np.clip(w, 0, NCOARSE - 1)


def _stream(s):
    return C.c_void_p(s.cuda_stream) if s is not None else C.c_void_p(torch.cuda.current_stream().cuda_stream)


class CoarseFeatures:
    """The coarse search that feeds the network, for one observation geometry.

    The band is brute-force dedispersed at COARSE_DMS coarse DMs over the
    search range (the full search's dedispersion kernel), downsampled 8x,
    detrended and normalised (the full search's preprocessing), then searched
    by the full search's FFA with periods 0.1-12.8 s at 48-64 bins.  The FFA
    peaks (S/N >= snr_floor) become a max-S/N map over NBINS log-period bins
    for each of the NCOARSE DM windows (the max over its coarse DMs).
    Features [NCOARSE][IN_CHANNELS][NBINS] bf16: the window's map and the
    zero-DM window's map (an RFI reference), as (S/N - floor)/10 clipped at 0.
    """

    def __init__(self, frequency_mhz, nsamples: int, tsamp: float, dm_max: float, device_id: int = 0,
                 snr_floor: float = 4.5):
        self.device = torch.device("cuda", device_id)
        freq = np.ascontiguousarray(frequency_mhz, np.float64)
        self.dm_max = dm_max
        self.snr_floor = snr_floor
        self.dm_step = dm_max / (COARSE_DMS - 1)
        self.program = core.DedispersionProgram(freq, nsamples, tsamp, 0.0, self.dm_step, COARSE_DMS,
                                                device_id=device_id)
        self.nout = self.program.nout
        self.tc = self.nout // DOWNSAMPLE
        self.tsamp_c = tsamp * DOWNSAMPLE
        self.stride = ((self.nout + 3) // 4) * 4
        self.stride_c = ((self.tc + 3) // 4) * 4
        self._series = torch.empty(COARSE_DMS * self.stride, dtype=torch.int32, device=self.device)
        self._coarse = torch.zeros((COARSE_DMS, self.stride_c), dtype=torch.float32, device=self.device)
        self.pre = core.PreprocessProgram(self.tc, self.tsamp_c, window_seconds=1.0, max_series=COARSE_DMS,
                                          device_id=device_id)
        plan = core.make_riptide_ffa_plan(self.tc, self.tsamp_c, 1.0 / F_MAX, 1.0 / F_MIN, bins_min=48,
                                          bins_max=64, duty_cycle_max=0.1)
        self.ffa = core.FfaProgram(plan, max_series=COARSE_DMS, device_id=device_id)
        self._prepared = torch.empty((COARSE_DMS, self.ffa.prepared_floats), dtype=torch.float32,
                                     device=self.device)

    def snr_map(self, filterbank: torch.Tensor) -> np.ndarray:
        """[NCOARSE][NBINS] max coarse FFA S/N per DM window and log-period bin."""
        lib = _lib.lib()
        s = torch.cuda.current_stream(self.device)
        staged = self.program.stage(filterbank)
        out = self.program.run(staged, 0, COARSE_DMS, out=self._series, out_stride=self.stride)
        check(lib.gf_prop_downsample(ptr(out), self.stride, COARSE_DMS, DOWNSAMPLE, self.tc, ptr(self._coarse),
                                     self.stride_c, _stream(s)))
        del staged
        stats = self.pre.run(self._coarse, COARSE_DMS)
        self.ffa.prepare(self._coarse, COARSE_DMS, stats, out=self._prepared)
        self.ffa.search_async(self._prepared, COARSE_DMS, self.snr_floor)
        peaks = self.ffa.expand(self.ffa.collect(self._prepared, COARSE_DMS, self.snr_floor))
        m = np.zeros((NCOARSE, NBINS), np.float32)
        if len(peaks):
            j = np.floor(BINS_PER_OCTAVE * np.log2(peaks["frequency"] / F_MIN)).astype(np.int64)
            w = window_of_dm(peaks["dm_index"].astype(np.float64) * self.dm_step, self.dm_max)
            ok = (j >= 0) & (j < NBINS)
            np.maximum.at(m, (w[ok], j[ok]), peaks["snr"][ok])
        return m

    def __call__(self, filterbank: torch.Tensor) -> torch.Tensor:
        """[NCOARSE][IN_CHANNELS][NBINS] bf16 features of a device-resident time-major filterbank."""
        m = np.clip((self.snr_map(filterbank) - self.snr_floor) / 10.0, 0.0, None)
        f = np.stack([m, np.broadcast_to(m[0], m.shape)], axis=1)
        return torch.from_numpy(np.ascontiguousarray(f)).to(self.device).to(torch.bfloat16)


class ProposalNet:
    """The network's fp32 master weights, bf16 copies, Adam state and the
    forward/backward passes through the library's kernels."""

    def __init__(self, device_id: int = 0, seed: int = 0):
        self.device = torch.device("cuda", device_id)
        g = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for cin, cout, k in LAYERS:
            std = math.sqrt(2.0 / (cin * k))
            self.w.append((torch.randn((cout, cin, k), generator=g) * std).to(self.device))
            self.b.append(torch.zeros(cout, device=self.device))
        c = LAYERS[-1][1]
        self.wh = (torch.randn(c, generator=g) * math.sqrt(1.0 / c)).to(self.device)
        self.bh = torch.full((1,), -3.0, device=self.device)
        self.params = self.w + self.b + [self.wh, self.bh]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.wb = [w.to(torch.bfloat16) for w in self.w]
        self.step = 0

    # -- persistence --------------------------------------------------------
    def state_dict(self) -> dict:
        return {f"p{i}": p.cpu() for i, p in enumerate(self.params)}

    def save(self, path, **meta) -> None:
        """Weights and metadata (numpy archive)."""
        arrays = {k: v.numpy() for k, v in self.state_dict().items()}
        arrays["meta"] = np.array(json.dumps(meta))
        np.savez(path, **arrays)

    def load(self, path) -> dict:
        """Loads weights saved by save(); returns the metadata."""
        z = np.load(path)
        self.load_state_dict({k: torch.from_numpy(z[k]) for k in z.files if k != "meta"})
        return json.loads(str(z["meta"])) if "meta" in z.files else {}

    def load_default(self) -> dict:
        """The model trained by `python -m gaffa_b200.proposal train` (shipped
        with the package)."""
        if not DEFAULT_WEIGHTS.exists():
            raise FileNotFoundError(str(DEFAULT_WEIGHTS))
        return self.load(DEFAULT_WEIGHTS)

    def load_state_dict(self, sd: dict) -> None:
        for i, p in enumerate(self.params):
            p.copy_(sd[f"p{i}"].to(self.device))
        self.wb = [w.to(torch.bfloat16) for w in self.w]

    # -- passes ---------------------------------------------------------------
    def forward(self, feat: torch.Tensor, keep: bool = False):
        """logits [B][OCTAVES] of features [B][IN_CHANNELS][NBINS] bf16."""
        lib = _lib.lib()
        s = _stream(None)
        B, L = feat.shape[0], feat.shape[2]
        acts = [feat.contiguous()]
        x = acts[0]
        for (cin, cout, k), wb, b in zip(LAYERS, self.wb, self.b):
            y = torch.empty((B, cout, L), dtype=torch.bfloat16, device=self.device)
            check(lib.gf_prop_conv_forward(ptr(x), ptr(wb), ptr(b), ptr(y), B, cin, cout, L, k, 1, s))
            acts.append(y)
            x = y
        logits = torch.empty((B, OCTAVES), dtype=torch.float32, device=self.device)
        check(lib.gf_prop_head(ptr(x), ptr(self.wh), ptr(self.bh), B, LAYERS[-1][1], L, OCTAVES, None, 0.0,
                               ptr(logits), None, None, None, None, s))
        return (logits, acts) if keep else logits

    def loss_and_grads(self, feat: torch.Tensor, labels: torch.Tensor, pos_weight: float):
        """Mean loss and the gradients of every parameter (same order as params)."""
        lib = _lib.lib()
        s = _stream(None)
        B, L = feat.shape[0], feat.shape[2]
        _, acts = self.forward(feat, keep=True)
        labels = labels.to(torch.float32).contiguous()
        grads = [torch.zeros_like(p) for p in self.params]
        nl = len(LAYERS)
        gw, gb, gwh, gbh = grads[:nl], grads[nl:2 * nl], grads[2 * nl], grads[2 * nl + 1]
        logits = torch.empty((B, OCTAVES), dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        dy = torch.empty((B, LAYERS[-1][1], L), dtype=torch.float32, device=self.device)
        check(lib.gf_prop_head(ptr(acts[-1]), ptr(self.wh), ptr(self.bh), B, LAYERS[-1][1], L, OCTAVES,
                               ptr(labels), pos_weight, ptr(logits), ptr(loss), ptr(dy), ptr(gwh), ptr(gbh), s))
        for i in range(nl - 1, -1, -1):
            cin, cout, k = LAYERS[i]
            dx = torch.empty((B, cin, L), dtype=torch.float32, device=self.device) if i > 0 else None
            check(lib.gf_prop_conv_backward(ptr(dy), ptr(acts[i + 1]), ptr(acts[i]), ptr(self.wb[i]),
                                            ptr(dx) if dx is not None else None, ptr(gw[i]), ptr(gb[i]), B, cin,
                                            cout, L, k, s))
            dy = dx
        scale = 1.0 / (B * OCTAVES)
        return float(loss.item()) * scale, [g * scale for g in grads], logits

    def train_step(self, feat, labels, pos_weight: float = 20.0, lr: float = 2e-3) -> float:
        lib = _lib.lib()
        s = _stream(None)
        loss, grads, _ = self.loss_and_grads(feat, labels, pos_weight)
        self.step += 1
        nl = len(LAYERS)
        for i, (p, g, m, v) in enumerate(zip(self.params, grads, self.m, self.v)):
            pb = self.wb[i] if i < nl else None
            check(lib.gf_prop_adam(ptr(p), ptr(g), ptr(m), ptr(v), ptr(pb) if pb is not None else None, p.numel(),
                                   lr, 0.9, 0.999, 1e-8, self.step, 1.0, s))
        return loss


HARMONIC_RATIOS = tuple(sorted({n / m for n in range(1, 5) for m in range(1, 5)}))


def injection_matches(candidates: np.ndarray, pulsar, observation_seconds: float, snr_min: float,
                      band_delay_per_dm: float) -> np.ndarray:
    """The candidates (S/N >= snr_min) that detect an injected pulsar: their
    frequency is within two Fourier bins (or 0.2 %) of the pulsar's times a
    harmonic ratio n/m (n, m <= 4), and their DM error smears the band by at
    most a quarter of the pulsar's period (band_delay_per_dm: seconds of
    band-crossing delay per unit DM)."""
    if not len(candidates):
        return candidates
    c = candidates[candidates["snr"] >= snr_min]
    if not len(c):
        return c
    f0 = 1.0 / pulsar.period
    ok = np.zeros(len(c), bool)
    for r in HARMONIC_RATIOS:
        tol = max(2.0 / observation_seconds, 2e-3 * r * f0)
        ok |= np.abs(c["frequency"] - r * f0) <= tol
    ok &= np.abs(c["dm"] - pulsar.dm) * band_delay_per_dm <= 0.25 * pulsar.period
    return c[ok]


def detected_injections(candidates: np.ndarray, pulsars, observation_seconds: float, snr_min: float,
                        band_delay_per_dm: float) -> list:
    """Per injected pulsar, the exhaustive-search candidates that detect it
    (empty: the exhaustive search missed it, so recall does not count it)."""
    return [injection_matches(candidates, p, observation_seconds, snr_min, band_delay_per_dm) for p in pulsars]


def labels_from_detections(pulsars, detections, dm_max: float) -> np.ndarray:
    """[NCOARSE][OCTAVES] 0/1: for every detected pulsar, its own window and
    octave and those of each candidate that detects it."""
    y = np.zeros((NCOARSE, OCTAVES), np.float32)
    for p, d in zip(pulsars, detections):
        if not len(d):
            continue
        y[window_of_dm(p.dm, dm_max), octave_of_period(p.period)] = 1.0
        y[window_of_dm(d["dm"], dm_max), octave_of_period(d["period"])] = 1.0
    return y


def labels_from_candidates(candidates: np.ndarray, dm_max: float, snr_min: float) -> np.ndarray:
    """[NCOARSE][OCTAVES] 0/1: windows and octaves holding a candidate."""
    y = np.zeros((NCOARSE, OCTAVES), np.float32)
    c = candidates[candidates["snr"] >= snr_min] if len(candidates) else candidates
    if len(c):
        y[window_of_dm(c["dm"], dm_max), octave_of_period(c["period"])] = 1.0
    return y


def baseline_scores(features: torch.Tensor) -> torch.Tensor:
    """The selection without the network: each window's largest coarse S/N
    ([NCOARSE][1], usable wherever logits are)."""
    return features[:, 0, :].float().max(dim=1, keepdim=True).values


def select_windows(logits: torch.Tensor, fraction: float) -> np.ndarray:
    """Indices of the top `fraction` of DM windows by their best octave logit."""
    score = logits.max(dim=1).values.float().cpu().numpy()
    k = max(1, int(math.ceil(fraction * len(score) - 1e-9)))
    return np.sort(np.argsort(-score, kind="stable")[:k])


def window_dm_indices(windows, ndm: int, dm_step: float, dm_max: float) -> np.ndarray:
    """Fine DM indices whose nearest window centre lies in `windows`."""
    fine = np.arange(ndm)
    return fine[np.isin(window_of_dm(fine * dm_step, dm_max), np.asarray(windows))]


def dm_ranges_for_windows(windows, ndm: int, dm_step: float, dm_max: float, granularity: int) -> list:
    """Contiguous [begin, end) DM-index ranges covering the windows' fine DMs,
    begins rounded down to the dedispersion granularity."""
    idx = window_dm_indices(windows, ndm, dm_step, dm_max)
    ranges = []
    for i in idx:
        b = (int(i) // granularity) * granularity
        if ranges and b <= ranges[-1][1]:
            ranges[-1][1] = max(ranges[-1][1], int(i) + 1)
        else:
            ranges.append([b, int(i) + 1])
    return [tuple(r) for r in ranges]


def recall(candidates: np.ndarray, windows, dm_max: float, snr_min: float) -> tuple[int, int]:
    """(found, total) exhaustive candidates with S/N >= snr_min inside the windows."""
    c = candidates[candidates["snr"] >= snr_min] if len(candidates) else candidates
    if not len(c):
        return 0, 0
    hit = np.isin(window_of_dm(c["dm"], dm_max), np.asarray(windows))
    return int(hit.sum()), len(c)


def injection_recall(detections, windows, dm_max: float) -> tuple[int, int]:
    """(found, total) over the injections the exhaustive search detected: an
    injection is found when a window holding one of its detecting candidates
    is searched (the restricted search repeats that candidate's DM trial)."""
    total = found = 0
    for d in detections:
        if not len(d):
            continue
        total += 1
        found += bool(np.isin(window_of_dm(d["dm"], dm_max), np.asarray(windows)).any())
    return found, total


@dataclasses.dataclass
class TrainingObservation:
    features: torch.Tensor        # [NCOARSE][IN_CHANNELS][NBINS] bf16 (device)
    labels: np.ndarray            # [NCOARSE][OCTAVES]
    candidates: np.ndarray        # exhaustive candidates (CAND_DTYPE)
    pulsars: list                 # the injections
    detections: list              # per injection, its detecting candidates


def synthetic_observation(seed: int, nchans: int, nsamples: int, tsamp: float, f_low: float, f_high: float,
                          dm_max: float, npulsars=(1, 4), snr=(5.0, 30.0), duty=(0.005, 0.1),
                          rfi_fraction: float = 0.3) -> synth.Observation:
    """Seeded training injection: P log-uniform 0.1-10 s, DM U(0, dm_max), duty
    0.5-10 %, folded S/N 5-30; a fraction with narrowband and impulsive RFI."""
    rng = np.random.default_rng(7_000_003 + seed)
    tobs = nsamples * tsamp
    pulsars = []
    for _ in range(int(rng.integers(npulsars[0], npulsars[1] + 1))):
        p = float(math.exp(rng.uniform(math.log(0.1), math.log(10.0))))
        d = float(rng.uniform(*duty))
        pulsars.append(synth.Pulsar(period=p, dm=float(rng.uniform(0.0, dm_max)), duty_cycle=d,
                                    amplitude=synth.folded_snr_amplitude(float(rng.uniform(*snr)), nchans, d, p,
                                                                         tobs, tsamp),
                                    phase=float(rng.uniform(0.0, 1.0))))
    rfi = synth.Rfi()
    if rng.random() < rfi_fraction:
        rfi = synth.Rfi(narrowband_fraction=0.05, narrowband_hz=50.0, impulse_hz=0.1)
    return synth.Observation(nchans=nchans, nsamples=nsamples, tsamp=tsamp, f_low=f_low, f_high=f_high, nbits=8,
                             seed=100_000 + seed, pulsars=pulsars, rfi=rfi)


def band_delay_per_dm(frequency_mhz) -> float:
    """Seconds of dispersion delay across the band per unit DM."""
    f = np.asarray(frequency_mhz, np.float64)
    return 4148.808 * abs(1.0 / f.min() ** 2 - 1.0 / f.max() ** 2)


def make_examples(cfg, seeds, snr_min: float | None = None, ds: search.DmSearch | None = None,
                  cf: CoarseFeatures | None = None, device_id: int = 0, **inject):
    """Features, injection-matched exhaustive-search labels and detections
    of seeded observations shaped like cfg."""
    obs0 = cfg.obs
    dm_max = cfg.dm_low + (cfg.ndm - 1) * cfg.dm_step
    ds = ds or search.from_config(cfg, device_id=device_id)
    cf = cf or CoarseFeatures(obs0.frequencies, obs0.nsamples, obs0.tsamp, dm_max, device_id=device_id)
    thr = cfg.snr_threshold if snr_min is None else snr_min
    bd = band_delay_per_dm(obs0.frequencies)
    tobs = obs0.nsamples * obs0.tsamp
    out = []
    for sd in seeds:
        obs = synthetic_observation(sd, obs0.nchans, obs0.nsamples, obs0.tsamp, obs0.f_low, obs0.f_high, dm_max,
                                    **inject)
        raw = core.synth_generate(obs, device_id=device_id)
        feat = cf(raw).clone()
        res = ds.run(raw)
        det = detected_injections(res.candidates, obs.pulsars, tobs, thr, bd)
        out.append(TrainingObservation(feat, labels_from_detections(obs.pulsars, det, dm_max), res.candidates,
                                       obs.pulsars, det))
        del raw
    return out, ds, cf


def train(net: ProposalNet, examples, epochs: int = 40, batch: int = 256, pos_weight: float = 10.0,
          lr: float = 1e-3, seed: int = 0) -> list:
    """Adam over all DM-window samples of the examples; returns the loss per epoch."""
    feats = torch.cat([e.features for e in examples])
    labels = torch.from_numpy(np.concatenate([e.labels for e in examples])).to(net.device)
    rng = np.random.default_rng(seed)
    history = []
    for _ in range(epochs):
        order = torch.from_numpy(rng.permutation(len(feats))).to(net.device)
        tot, n = 0.0, 0
        for i in range(0, len(order), batch):
            idx = order[i:i + batch]
            tot += net.train_step(feats[idx], labels[idx], pos_weight, lr) * len(idx)
            n += len(idx)
        history.append(tot / n)
    return history


def evaluate(scorer, examples, fractions, dm_max: float) -> dict:
    """Injection recall at each window fraction: {fraction: (found, total)}."""
    out = {}
    for frac in fractions:
        found = total = 0
        for e in examples:
            f, t = injection_recall(e.detections, select_windows(scorer(e), frac), dm_max)
            found += f
            total += t
        out[frac] = (found, total)
    return out


def evaluate_held_out(cfg, nobs: int, seed: int, dm_max: float, coarse_cost: float | None) -> dict:
    """Recall of the shipped weights, the max-coarse-S/N heuristic and random
    windows on nobs held-out seeded observations (seeds 20000 + seed + i, never
    used for training or validation), at every window fraction, with the
    speed-up over the exhaustive search that each fraction implies:
    1 / (coarse_cost + fraction).  coarse_cost defaults to the measured cost
    of the coarse search and network on the first observation."""
    import time
    held, ds, cf = make_examples(cfg, range(20_000 + seed, 20_000 + seed + nobs))
    net = ProposalNet()
    meta = net.load_default()
    if coarse_cost is None:
        obs = synthetic_observation(20_000 + seed, cfg.obs.nchans, cfg.obs.nsamples, cfg.obs.tsamp, cfg.obs.f_low,
                                    cfg.obs.f_high, dm_max)
        raw = core.synth_generate(obs)
        ds.run(raw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ds.run(raw)
        torch.cuda.synchronize()
        t_full = time.perf_counter() - t0
        t0 = time.perf_counter()
        net.forward(cf(raw))
        torch.cuda.synchronize()
        coarse_cost = (time.perf_counter() - t0) / t_full
    fractions = [k / NCOARSE for k in range(1, NCOARSE + 1)]
    rec = evaluate(lambda e: net.forward(e.features), held, fractions, dm_max)
    base = evaluate(lambda e: baseline_scores(e.features), held, fractions, dm_max)
    rng = np.random.default_rng(seed)
    rand = evaluate(lambda e: torch.from_numpy(rng.random((NCOARSE, 1))), held, fractions, dm_max)
    curve = {f"{f:.4f}": {"speedup": 1.0 / (coarse_cost + f), "trained": rec[f], "heuristic": base[f],
                          "random": rand[f]} for f in fractions}
    out = {"held_out_observations": nobs, "detected_injections": rec[fractions[-1]][1],
           "coarse_cost": coarse_cost, "weights": meta.get("trained_on", ""), "curve": curve}
    print(json.dumps(out), flush=True)
    return out


def main() -> None:
    """python -m gaffa_b200.proposal train [--train N] [--val M] [--nsamples-log2 L] [--epochs E] [--out PATH]
    python -m gaffa_b200.proposal evaluate [--val M]   (held-out recall curve of the shipped weights)

    Generates seeded survey-band injections (4096 channels, 1100-1700 MHz,
    DMs 0-1000 in 2048 trials, 2^L samples), labels them with the exhaustive
    search, trains the network on the GPU with the library's kernels, and
    stores the weights with the smallest window fraction that keeps >= 99 %
    injection recall on the validation observations (or all windows)."""
    import argparse
    import time

    from . import configs
    ap = argparse.ArgumentParser()
    ap.add_argument("command", choices=["train", "evaluate"])
    ap.add_argument("--train", type=int, default=100)
    ap.add_argument("--val", type=int, default=20)
    ap.add_argument("--nsamples-log2", type=int, default=20)
    ap.add_argument("--epochs", type=int, default=80)
    ap.add_argument("--pos-weight", type=float, default=10.0)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--coarse-cost", type=float, default=None,
                    help="evaluate: cost of the coarse search and network as a fraction of the exhaustive search")
    a = ap.parse_args()
    cfg = configs.survey_size(nsamples=1 << a.nsamples_log2)
    dm_max = cfg.dm_low + (cfg.ndm - 1) * cfg.dm_step
    if a.command == "evaluate":
        evaluate_held_out(cfg, a.val, a.seed, dm_max, a.coarse_cost)
        return
    t0 = time.time()
    train_set, ds, cf = make_examples(cfg, range(a.seed, a.seed + a.train))
    val_set, _, _ = make_examples(cfg, range(10_000 + a.seed, 10_000 + a.seed + a.val), ds=ds, cf=cf)
    t1 = time.time()
    net = ProposalNet(seed=a.seed)
    history = train(net, train_set, epochs=a.epochs, pos_weight=a.pos_weight, lr=a.lr, seed=a.seed)
    fractions = [k / NCOARSE for k in range(1, NCOARSE + 1)]
    rec = evaluate(lambda e: net.forward(e.features), val_set, fractions, dm_max)
    base = evaluate(lambda e: baseline_scores(e.features), val_set, fractions, dm_max)
    rng = np.random.default_rng(a.seed)
    rand = evaluate(lambda e: torch.from_numpy(rng.random((NCOARSE, 1))), val_set, fractions, dm_max)
    chosen = next((f for f in fractions if rec[f][1] and rec[f][0] >= 0.99 * rec[f][1]), 1.0)
    report = {f"{f:.4f}": {"trained": rec[f], "heuristic": base[f], "random": rand[f]} for f in fractions[1::2]}
    meta = {"fraction": chosen, "trained_on": f"{a.train} seeded survey-band injections, 2^{a.nsamples_log2} samples",
            "epochs": a.epochs, "pos_weight": a.pos_weight, "lr": a.lr, "final_loss": history[-1],
            "val_observations": a.val, "val_recall_at_fraction": rec[chosen],
            "heuristic_recall_at_fraction": base[chosen], "examples_seconds": t1 - t0, "val_curve": report}
    net.save(a.out, **meta)
    print(json.dumps({"meta": meta}), flush=True)


if __name__ == "__main__":
    main()
