"""Seeded synthetic filterbanks with injected pulsars and RFI.

The reference ships no generator (its tests use small arithmetic patterns), so
this module defines one.  Every sample is a pure function of
``(seed, time, channel)``, so the numpy implementation here and the CUDA
generator in ``csrc/synth.cu`` produce the same noise bit for bit; the
injected pulse amplitudes are computed in float64 on both sides.

Noise model: ``128 + 16 z`` where ``z`` is an Irwin-Hall(12) deviate built from
twelve 16-bit words of a splitmix64 stream (exactly mean 0, variance 1,
support +-6).  The value is rounded and clipped to uint8.  For 2-bit data the
same deviate is thresholded at the N(0,1) quartiles (levels 0..3).

Channel order is frequency-ascending (``freq[-1]`` is the highest channel and the
dedispersion reference frequency), which is the order gaffa's filterbank reader
produces by default after reversing a descending file.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

DISPERSION_CONSTANT = 4148.808  # s MHz^2 (cold-plasma delay constant)

_M64 = (1 << 64) - 1
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_MIX1 = np.uint64(0xBF58476D1CE4E5B9)
_MIX2 = np.uint64(0x94D049BB133111EB)
# N(0,1) quartiles scaled by 4096 (deviates are held in 1/4096 units)
_Q_LO = -2763  # round(-0.6744897501960817 * 4096)
_Q_HI = 2763


@dataclasses.dataclass
class Pulsar:
    period: float          # seconds
    dm: float              # pc cm^-3
    duty_cycle: float      # FWHM / period
    amplitude: float       # peak counts per channel (noise sd is 16)
    phase: float = 0.25    # pulse centre phase at t = 0 (top of the band)


@dataclasses.dataclass
class Rfi:
    narrowband_fraction: float = 0.0   # fraction of channels modulated
    narrowband_hz: float = 50.0        # sinusoidal modulation frequency
    narrowband_amplitude: float = 24.0 # counts
    impulse_hz: float = 0.0            # zero-DM impulse rate (0 disables)
    impulse_amplitude: float = 48.0    # counts, all channels, one sample wide


@dataclasses.dataclass
class Observation:
    nchans: int
    nsamples: int
    tsamp: float
    f_low: float
    f_high: float
    nbits: int = 8
    seed: int = 0
    pulsars: list = dataclasses.field(default_factory=list)
    rfi: Rfi = dataclasses.field(default_factory=Rfi)

    @property
    def frequencies(self) -> np.ndarray:
        return channel_frequencies(self.nchans, self.f_low, self.f_high)

    @property
    def ref_frequency(self) -> float:
        return float(self.frequencies.max())


def channel_frequencies(nchans: int, f_low: float, f_high: float) -> np.ndarray:
    """Ascending channel centre frequencies spanning [f_low, f_high] in MHz."""
    if nchans == 1:
        return np.array([f_high], np.float64)
    return f_low + (f_high - f_low) * np.arange(nchans, dtype=np.float64) / (nchans - 1)


def _splitmix(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _MIX1
        z = (z ^ (z >> np.uint64(27))) * _MIX2
        return z ^ (z >> np.uint64(31))


def noise_units(seed: int, index: np.ndarray) -> np.ndarray:
    """Irwin-Hall(12) deviates in 1/4096 units, i.e. round(4096 z) = S/16 - 24576.

    ``index`` is the flat sample index ``t * nchans + c``.  Returns int64 ``S``
    (sum of twelve 16-bit words); ``z = S / 65536 - 6``.
    """
    base = (np.uint64(seed & 0xFFFFF) << np.uint64(44)) ^ (index.astype(np.uint64) * np.uint64(3))
    s = np.zeros(index.shape, np.int64)
    for k in range(3):
        h = _splitmix(base + np.uint64(k))
        for j in range(4):
            s += ((h >> np.uint64(16 * j)) & np.uint64(0xFFFF)).astype(np.int64)
    return s


def pulse_units(obs: Observation, t: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Injected signal (pulsars + RFI) in 1/4096 counts, rounded to int64."""
    freq = obs.frequencies
    fref = obs.ref_frequency
    total = np.zeros(np.broadcast(t, c).shape, np.float64)
    tt = t.astype(np.float64) * obs.tsamp
    for p in obs.pulsars:
        delay = DISPERSION_CONSTANT * p.dm * (1.0 / freq[c] ** 2 - 1.0 / fref ** 2)
        ph = (tt - delay) / p.period - p.phase
        ph = ph - np.floor(ph + 0.5)
        sigma = p.duty_cycle / 2.3548200450309493
        x = ph / sigma
        total += np.where(np.abs(x) < 12.0, p.amplitude * np.exp(-0.5 * (x * x)), 0.0)
    r = obs.rfi
    if r.narrowband_fraction > 0.0:
        nb = _narrowband_mask(obs)[c]
        total += np.where(nb, r.narrowband_amplitude * np.sin(2.0 * math.pi * r.narrowband_hz * tt), 0.0)
    if r.impulse_hz > 0.0:
        period_samples = max(1, int(round(1.0 / (r.impulse_hz * obs.tsamp))))
        total += np.where(t % period_samples == period_samples // 2, r.impulse_amplitude, 0.0)
    return np.rint(total * 4096.0).astype(np.int64)


def _narrowband_mask(obs: Observation) -> np.ndarray:
    n = int(round(obs.rfi.narrowband_fraction * obs.nchans))
    idx = (_splitmix(np.arange(obs.nchans, dtype=np.uint64) + np.uint64(obs.seed * 7919 + 17))
           % np.uint64(1 << 30)).astype(np.int64)
    order = np.argsort(idx, kind="stable")
    mask = np.zeros(obs.nchans, bool)
    mask[order[:n]] = True
    return mask


def generate(obs: Observation, t_begin: int = 0, t_end: int | None = None) -> np.ndarray:
    """Samples for times [t_begin, t_end) as uint8 [time][channel].

    8-bit data holds ``clip(round(128 + 16 z + signal), 0, 255)``; 2-bit data holds
    the quartile level of ``z + signal / 16`` (use :func:`pack_2bit` to pack).
    """
    t_end = obs.nsamples if t_end is None else t_end
    t = np.arange(t_begin, t_end, dtype=np.int64)[:, None]
    c = np.arange(obs.nchans, dtype=np.int64)[None, :]
    s = noise_units(obs.seed, t * obs.nchans + c)
    sig = pulse_units(obs, t, c)
    if obs.nbits == 8:
        # value = 32 + S/4096 + signal/4096, rounded half up, clipped
        v = (32 * 4096 + s + sig + 2048) >> 12
        return np.clip(v, 0, 255).astype(np.uint8)
    if obs.nbits == 2:
        # z*4096 = S/16 - 24576 ; signal in counts / 16 = deviate units
        zu = (s >> 4) - 24576 + (sig >> 4)
        lvl = (zu >= _Q_LO).astype(np.uint8) + (zu >= 0).astype(np.uint8) + (zu >= _Q_HI).astype(np.uint8)
        return lvl
    raise ValueError("nbits must be 8 or 2")


def pack_2bit(levels: np.ndarray) -> np.ndarray:
    """Pack [time][channel] 2-bit levels, channel 4k+j into bits [2j, 2j+1] of byte k."""
    t, c = levels.shape
    if c % 4:
        raise ValueError("2-bit packing needs nchans % 4 == 0")
    lv = levels.reshape(t, c // 4, 4).astype(np.uint8)
    return (lv[..., 0] | (lv[..., 1] << 2) | (lv[..., 2] << 4) | (lv[..., 3] << 6)).astype(np.uint8)


def unpack_2bit(packed: np.ndarray, nchans: int) -> np.ndarray:
    t = packed.shape[0]
    out = np.empty((t, nchans), np.uint8)
    for j in range(4):
        out[:, j::4] = (packed >> (2 * j)) & 3
    return out


def folded_snr_amplitude(target_snr: float, nchans: int, duty: float, period: float,
                         tobs: float, tsamp: float, noise_sd: float = 16.0) -> float:
    """Per-channel peak amplitude giving roughly ``target_snr`` after folding.

    Matched-filter estimate for a Gaussian pulse: S/N = A sqrt(nchans W N) / sd,
    with W = 1.064 FWHM in samples and N periods in the observation.
    """
    w = 1.0645 * duty * period / tsamp
    n = tobs / period
    return target_snr * noise_sd / math.sqrt(nchans * w * n)
