"""Learned DM/period proposal in front of the exhaustive search.

The coarse view of an observation is its band split into 32 subbands,
brute-force dedispersed at 64 coarse DMs over the search range (the same
dedispersion kernel as the full search, on channel ranges) and downsampled
16x.  For every (coarse DM, subband) series the power spectrum (cuFFT through
torch.fft) feeds the harmonic-sum feature kernel, giving a [64][32][448]
bf16 map: 7 period octaves (0.1-12.8 s) x 64 log-frequency bins.  A small
1-D convolutional network (csrc/proposal.cu: 32-64-64-32 channels, kernel 9,
then a per-bin score pooled per octave) turns each coarse DM's [32][448]
map into 7 octave logits.

Training labels come from the exhaustive search's own candidates (S/N above
the search threshold) on seeded synthetic injections: a coarse DM window and
period octave holding a candidate is positive.  At inference the windows are
ranked by their best octave score and only the top fraction goes to the
full-resolution search; the exhaustive search remains the fallback and the
judge of recall.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math

import numpy as np
import torch

from . import _lib, core, search, synth
from ._lib import check, ptr

OCTAVES = 7
BINS_PER_OCTAVE = 64
NBINS = OCTAVES * BINS_PER_OCTAVE
F_MAX = 10.0                         # Hz: period 0.1 s
F_MIN = F_MAX / 2 ** OCTAVES         # Hz: period 12.8 s
NSUB = 32
NCOARSE = 64
DOWNSAMPLE = 16
LAYERS = ((32, 64, 9), (64, 64, 9), (64, 32, 9))


def bin_edges() -> np.ndarray:
    """Log-frequency bin edges (Hz), ascending: bin j spans one 64th of an octave."""
    return (F_MIN * 2.0 ** (np.arange(NBINS + 1) / BINS_PER_OCTAVE)).astype(np.float32)


def octave_of_period(period) -> np.ndarray:
    """Octave index (0 = 6.4-12.8 s ... 6 = 0.1-0.2 s), clipped to the grid."""
    f = 1.0 / np.asarray(period, dtype=np.float64)
    j = np.floor(BINS_PER_OCTAVE * np.log2(f / F_MIN)).astype(np.int64)
    return np.clip(j // BINS_PER_OCTAVE, 0, OCTAVES - 1)


def window_of_dm(dm, dm_max: float) -> np.ndarray:
    """Coarse DM window (nearest of the NCOARSE coarse DMs over [0, dm_max])."""
    w = np.rint(np.asarray(dm, dtype=np.float64) / dm_max * (NCOARSE - 1)).astype(np.int64)
    return np.clip(w, 0, NCOARSE - 1)


def _stream(s):
    return C.c_void_p(s.cuda_stream) if s is not None else C.c_void_p(torch.cuda.current_stream().cuda_stream)


class CoarseFeatures:
    """Coarse subband dedispersion + spectral features of one observation geometry."""

    def __init__(self, frequency_mhz, nsamples: int, tsamp: float, dm_max: float, device_id: int = 0):
        self.device = torch.device("cuda", device_id)
        freq = np.ascontiguousarray(frequency_mhz, np.float64)
        nchans = len(freq)
        if nchans % NSUB:
            raise ValueError(f"nchans must be a multiple of {NSUB}")
        sbc = nchans // NSUB
        self.dm_max = dm_max
        self.tsamp = tsamp
        self.programs = [core.DedispersionProgram(freq, nsamples, tsamp, 0.0, dm_max / (NCOARSE - 1), NCOARSE,
                                                  ref_frequency_mhz=float(freq.max()), chan_begin=s * sbc,
                                                  chan_end=(s + 1) * sbc, device_id=device_id)
                         for s in range(NSUB)]
        self.nout = min(p.nout for p in self.programs)
        self.t16 = self.nout // DOWNSAMPLE
        self.stride = ((max(p.nout for p in self.programs) + 3) // 4) * 4
        self._series = torch.empty(NCOARSE * self.stride, dtype=torch.int32, device=self.device)
        self._coarse = torch.empty((NCOARSE * NSUB, self.t16), dtype=torch.float32, device=self.device)
        self._edges = torch.from_numpy(bin_edges()).to(self.device)
        self.df = 1.0 / (self.t16 * DOWNSAMPLE * tsamp)

    def __call__(self, filterbank: torch.Tensor) -> torch.Tensor:
        """[NCOARSE][NSUB][NBINS] bf16 features of a device-resident time-major filterbank."""
        lib = _lib.lib()
        s = torch.cuda.current_stream(self.device)
        for sb, prog in enumerate(self.programs):
            staged = prog.stage(filterbank)
            out = prog.run(staged, 0, NCOARSE, out=self._series, out_stride=self.stride)
            # rows dm of this subband -> coarse[dm * NSUB + sb]
            dst = self._coarse.view(-1)[sb * self.t16:]
            check(lib.gf_prop_downsample(ptr(out), self.stride, NCOARSE, DOWNSAMPLE, self.t16, ptr(dst),
                                         NSUB * self.t16, _stream(s)))
        x = self._coarse
        x = (x - x.mean(dim=1, keepdim=True)) / x.std(dim=1, keepdim=True).clamp_min(1e-6)
        spec = torch.fft.rfft(x, dim=1)
        power = spec.real.square() + spec.imag.square()
        power[:, 0] = 0.0
        power /= power[:, 1:].mean(dim=1, keepdim=True).clamp_min(1e-12)
        power = power.contiguous()
        feat = torch.empty((NCOARSE * NSUB, NBINS), dtype=torch.bfloat16, device=self.device)
        check(lib.gf_prop_features(ptr(power), power.shape[0], power.shape[1], self.df, ptr(self._edges), NBINS,
                                   ptr(feat), _stream(s)))
        return feat.view(NCOARSE, NSUB, NBINS)


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

    def load_state_dict(self, sd: dict) -> None:
        for i, p in enumerate(self.params):
            p.copy_(sd[f"p{i}"].to(self.device))
        self.wb = [w.to(torch.bfloat16) for w in self.w]

    # -- passes ---------------------------------------------------------------
    def forward(self, feat: torch.Tensor, keep: bool = False):
        """logits [B][OCTAVES] of features [B][32][NBINS] bf16."""
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


def labels_from_candidates(candidates: np.ndarray, dm_max: float, snr_min: float) -> np.ndarray:
    """[NCOARSE][OCTAVES] 0/1: windows and octaves holding a candidate."""
    y = np.zeros((NCOARSE, OCTAVES), np.float32)
    c = candidates[candidates["snr"] >= snr_min] if len(candidates) else candidates
    if len(c):
        y[window_of_dm(c["dm"], dm_max), octave_of_period(c["period"])] = 1.0
    return y


def select_windows(logits: torch.Tensor, fraction: float) -> np.ndarray:
    """Indices of the top `fraction` of coarse DM windows by their best octave logit."""
    score = logits.max(dim=1).values.float().cpu().numpy()
    k = max(1, int(math.ceil(fraction * len(score))))
    return np.sort(np.argsort(-score, kind="stable")[:k])


def window_dm_indices(windows, ndm: int, dm_step: float, dm_max: float) -> np.ndarray:
    """Fine DM indices whose nearest coarse DM lies in `windows`."""
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


@dataclasses.dataclass
class TrainingObservation:
    features: torch.Tensor        # [NCOARSE][NSUB][NBINS] bf16 (device)
    labels: np.ndarray            # [NCOARSE][OCTAVES]
    candidates: np.ndarray        # exhaustive candidates (CAND_DTYPE)


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


def make_examples(cfg, seeds, snr_min: float | None = None, ds: search.DmSearch | None = None,
                  cf: CoarseFeatures | None = None, device_id: int = 0, **inject):
    """Features and exhaustive-search labels of seeded observations shaped like cfg."""
    obs0 = cfg.obs
    dm_max = cfg.dm_low + (cfg.ndm - 1) * cfg.dm_step
    ds = ds or search.from_config(cfg, device_id=device_id)
    cf = cf or CoarseFeatures(obs0.frequencies, obs0.nsamples, obs0.tsamp, dm_max, device_id=device_id)
    thr = cfg.snr_threshold if snr_min is None else snr_min
    out = []
    for sd in seeds:
        obs = synthetic_observation(sd, obs0.nchans, obs0.nsamples, obs0.tsamp, obs0.f_low, obs0.f_high, dm_max,
                                    **inject)
        raw = core.synth_generate(obs, device_id=device_id)
        feat = cf(raw).clone()
        res = ds.run(raw)
        out.append(TrainingObservation(feat, labels_from_candidates(res.candidates, dm_max, thr), res.candidates))
        del raw
    return out, ds, cf


def train(net: ProposalNet, examples, epochs: int = 40, batch: int = 256, pos_weight: float = 20.0,
          lr: float = 2e-3, seed: int = 0) -> list:
    """Adam over all coarse-DM samples of the examples; returns the loss per epoch."""
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
