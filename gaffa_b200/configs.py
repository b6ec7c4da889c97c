"""Named workloads: the observation shapes and search settings of the
benchmark configurations (plain end-to-end, survey-size, wide-range subband,
batched uneven, learned proposal), plus scaled-down variants for tests.

All inputs are synthetic and seeded (``synth.py``); no dataset is involved.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import synth


@dataclasses.dataclass
class SearchConfig:
    name: str
    obs: synth.Observation
    dm_low: float
    dm_step: float
    ndm: int
    period_min: float
    period_max: float
    bins_min: int = 180
    bins_max: int = 256
    duty_cycle_max: float = 0.2
    width_trials: tuple | None = None      # explicit widths (None = plan generator)
    window_seconds: float = 1.0            # running-median detrend window
    min_points: int = 101
    snr_threshold: float = 8.0
    fold_nbin: int = 64
    dedispersion: str = "brute"            # "brute" | "subband"
    subband_channels: int = 64
    ndm_per_nominal: int = 32
    frequency_cluster_radius: float = 0.1
    dm_cluster_radius: int = 1
    device_candidates: bool = False        # select candidates on the device (10^7+ raw peaks)

    @property
    def dms(self) -> np.ndarray:
        return self.dm_low + np.arange(self.ndm, dtype=np.float64) * self.dm_step

    def plan_options(self) -> dict:
        return dict(period_min=self.period_min, period_max=self.period_max,
                    bins_min=self.bins_min, bins_max=self.bins_max,
                    duty_cycle_max=self.duty_cycle_max)

    def preprocess_options(self) -> dict:
        return dict(window_seconds=self.window_seconds, min_points=self.min_points,
                    normalise=True, reject_constant=True)


def plain_end_to_end(seed: int = 0, nsamples: int = 1 << 18, nchans: int = 256,
                     ndm: int = 512) -> SearchConfig:
    """256 ch over 1200-1500 MHz, uint8, 64 us, 2^18 samples, one pulsar
    (P 0.5 s, DM 100, FWHM 2 %, 2 sd per channel); 512 DMs over 0-200;
    1 s running median; FFA 0.2-2 s; widths 1..32; fold into 64 bins."""
    obs = synth.Observation(
        nchans=nchans, nsamples=nsamples, tsamp=64e-6, f_low=1200.0, f_high=1500.0,
        nbits=8, seed=seed,
        pulsars=[synth.Pulsar(period=0.5, dm=100.0, duty_cycle=0.02, amplitude=32.0)])
    return SearchConfig(
        name="plain_end_to_end", obs=obs, dm_low=0.0, dm_step=200.0 / (ndm - 1),
        ndm=ndm, period_min=0.2, period_max=2.0, width_trials=(1, 2, 4, 8, 16, 32))


def _survey_pulsars(rng: np.random.Generator, count: int, nchans: int, tobs: float,
                    tsamp: float, dm_max: float, duty=(0.01, 0.05), snr=(8.0, 30.0),
                    periods=(0.1, 10.0)) -> list:
    out = []
    for _ in range(count):
        p = float(math.exp(rng.uniform(math.log(periods[0]), math.log(periods[1]))))
        d = float(rng.uniform(duty[0], duty[1]))
        target = float(rng.uniform(*snr))
        out.append(synth.Pulsar(
            period=p, dm=float(rng.uniform(0.0, dm_max)), duty_cycle=d,
            amplitude=synth.folded_snr_amplitude(target, nchans, d, p, tobs, tsamp),
            phase=float(rng.uniform(0.0, 1.0))))
    return out


def survey_size(seed: int = 0, nsamples: int = 1 << 23, nchans: int = 4096,
                ndm: int = 2048) -> SearchConfig:
    """4096 ch over 1100-1700 MHz, uint8, 64 us, 2^23 samples, 8 pulsars
    (P log-uniform 0.1-10 s, DM U(0,1000), duty 1-5 %, folded S/N 8-30);
    2048 DMs over 0-1000; FFA 0.1-10 s with widths up to 10 % duty."""
    tsamp = 64e-6
    rng = np.random.default_rng(1_000_003 + seed)
    obs = synth.Observation(
        nchans=nchans, nsamples=nsamples, tsamp=tsamp, f_low=1100.0, f_high=1700.0,
        nbits=8, seed=seed,
        pulsars=_survey_pulsars(rng, 8, nchans, nsamples * tsamp, tsamp, 1000.0))
    return SearchConfig(
        name="survey_size", obs=obs, dm_low=0.0, dm_step=1000.0 / (ndm - 1), ndm=ndm,
        period_min=0.1, period_max=10.0, duty_cycle_max=0.1)


def wide_subband(seed: int = 0, nsamples: int = 1 << 22, nchans: int = 4096,
                 ndm: int = 8192) -> SearchConfig:
    """2-bit packed, 4096 ch over 300-400 MHz, 81.92 us, 2^22 samples, 64
    subbands, nominal subband DMs every 20, 8192 DMs over 0-3000, 16 pulsars,
    5 % narrowband 50 Hz RFI channels and 0.1 Hz zero-DM impulses."""
    tsamp = 81.92e-6
    rng = np.random.default_rng(2_000_003 + seed)
    dm_step = 3000.0 / (ndm - 1)
    obs = synth.Observation(
        nchans=nchans, nsamples=nsamples, tsamp=tsamp, f_low=300.0, f_high=400.0,
        nbits=2, seed=seed,
        pulsars=_survey_pulsars(rng, 16, nchans, nsamples * tsamp, tsamp, 3000.0),
        rfi=synth.Rfi(narrowband_fraction=0.05, narrowband_hz=50.0, impulse_hz=0.1))
    return SearchConfig(
        name="wide_subband", obs=obs, dm_low=0.0, dm_step=dm_step, ndm=ndm,
        period_min=0.1, period_max=10.0, duty_cycle_max=0.1, dedispersion="subband",
        subband_channels=nchans // 64, ndm_per_nominal=int(math.ceil(20.0 / dm_step)),
        device_candidates=True)


def batched_uneven(seed: int = 0, nobs: int = 64, nchans_choices=(1024, 2048, 4096), log2_nsamples=(20.0, 23.0),
                   ndm_range=(256, 4096), dm_max: float = 1000.0, max_pulsars: int = 4) -> list:
    """64 independent observations of uneven geometry: channels from
    {1024, 2048, 4096} over 1200-1500 MHz, uint8, 64 us, lengths log-uniform
    over 2^20-2^23 samples, 256-4096 DM trials over 0-dm_max, an FFA period
    range drawn inside 0.1-10 s and 0-4 injected pulsars each (folded S/N
    8-30, duty 1-5 %).  Observation i uses seed seed * 1000 + i.  The
    keyword ranges give scaled-down batches of the same laws."""
    tsamp = 64e-6
    rng = np.random.default_rng(3_000_003 + seed)
    out = []
    for i in range(nobs):
        nchans = int(rng.choice(nchans_choices))
        nsamples = int(round(2.0 ** rng.uniform(*log2_nsamples) / 16.0)) * 16
        ndm = int(rng.integers(ndm_range[0], ndm_range[1] + 1))
        p_lo = float(math.exp(rng.uniform(math.log(0.1), math.log(1.0))))
        p_hi = float(min(10.0, p_lo * math.exp(rng.uniform(math.log(2.0), math.log(100.0)))))
        npsr = int(rng.integers(0, max_pulsars + 1))
        obs = synth.Observation(
            nchans=nchans, nsamples=nsamples, tsamp=tsamp, f_low=1200.0, f_high=1500.0, nbits=8,
            seed=seed * 1000 + i,
            pulsars=_survey_pulsars(rng, npsr, nchans, nsamples * tsamp, tsamp, dm_max, periods=(p_lo, p_hi)))
        out.append(SearchConfig(
            name=f"batched_uneven_{i}", obs=obs, dm_low=0.0, dm_step=dm_max / (ndm - 1), ndm=ndm,
            period_min=p_lo, period_max=p_hi, duty_cycle_max=0.1))
    return out


CONFIGS = {
    "plain_end_to_end": plain_end_to_end,
    "survey_size": survey_size,
    "wide_subband": wide_subband,
}
