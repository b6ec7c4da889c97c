"""gaffa's compiled-module surface (``gaffa._core``) on the B200 path.

Same names, keyword arguments, defaults, result classes and error types as the
reference's pybind module (python/gaffa/_core.pyi; bindings in
src/gaffa/python/{dedispersion,ffa,folding,filterbank}_bindings.cpp), so code
written against ``gaffa._core`` -- or the public ``gaffa.dedispersion``,
``gaffa.ffa``, ``gaffa.io`` and ``gaffa.pfold`` modules mirrored beside this
one -- runs here unchanged.  Every computation is a call into
libgaffa_b200.so through gaffa_b200.core.

Two deliberate differences, both loud:
* ``backend`` defaults to ``"cuda"`` and ``backend="cpu"`` raises ValueError:
  this library is the CUDA path only and never falls back to a CPU.
* Dedispersion takes 8-bit filterbanks (the sample type of the search path);
  16-bit and float32 filterbanks raise TypeError, except in
  ``dedisperse_spectrum``, which takes all three like the reference.
"""
from __future__ import annotations

import enum
import math
from pathlib import Path

import numpy as np

from .. import _lib, core

__all__ = [
    "ChannelOrderPolicy", "ReverseBackend", "FilterbankHeader", "Filterbank", "DedispersedResult",
    "DedispersedSpectrum", "FoldResult", "FfaPlan", "FfaPeak", "FoldedProfile", "_make_riptide_ffa_plan",
    "_ffa_search_cpu", "_ffa_search_cuda_host", "_fold_dedispersed_profile", "_fold_dedispersed_spectrum",
    "dedisperse_spectrum", "dedisperse_single_dm", "dedisperse_multi_dm", "dedisperse_subband",
    "cuda_device_count", "cuda_runtime_version",
]

CPU_BACKEND_MESSAGE = ("gaffa_b200 is the CUDA path only: backend='cpu' is not provided "
                       "(use backend='cuda')")


# ---------------------------------------------------------------------------
# runtime
# ---------------------------------------------------------------------------

def cuda_device_count() -> int:
    """Visible CUDA devices (cuda_device_count, src/gaffa/vector_add.cu:81-89)."""
    import ctypes as C
    n = C.c_int32()
    _lib.check(_lib.lib().gf_cuda_device_count(C.byref(n)))
    return int(n.value)


def cuda_runtime_version() -> int:
    """CUDA runtime version, e.g. 12090 (src/gaffa/vector_add.cu:75-79)."""
    import ctypes as C
    v = C.c_int32()
    _lib.check(_lib.lib().gf_cuda_runtime_version(C.byref(v)))
    return int(v.value)


def _backend(value: str) -> None:
    """parse_backend (dedispersion_bindings.cpp:55-64), CUDA only."""
    if value == "cuda":
        return
    if value == "cpu":
        raise ValueError(CPU_BACKEND_MESSAGE)
    raise ValueError(f"unknown dedispersion backend: {value}")


def _device(device_id: int) -> int:
    if not isinstance(device_id, (int, np.integer)) or device_id < 0:
        raise ValueError("device_id must be non-negative")
    return int(device_id)


# ---------------------------------------------------------------------------
# filterbank (filterbank_bindings.cpp, include/gaffa/filterbank.h)
# ---------------------------------------------------------------------------

class ChannelOrderPolicy(enum.Enum):
    FrequencyAscending = "frequency_ascending"
    PreserveFileOrder = "preserve_file_order"


class ReverseBackend(enum.Enum):
    Auto = "auto"
    CpuScalar = "cpu_scalar"
    CpuOpenmp = "cpu_openmp"


_HEADER_INT = ("header_size", "nsamples", "telescope_id", "machine_id", "data_type", "barycentric",
               "pulsarcentric", "ibeam", "nbeams", "npuls", "nbins", "nbits", "nifs", "nchans")
_HEADER_FLOAT = ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "fch1", "foff", "refdm",
                 "period")


class FilterbankHeader:
    """Parsed SIGPROC header (FilterbankHeader, include/gaffa/filterbank.h);
    frequency_table is aligned with Filterbank.data's channel axis."""

    def __init__(self, fields: dict | None = None, frequency_table=None):
        fields = fields or {}
        for k in _HEADER_INT:
            setattr(self, k, int(fields.get(k, 0)))
        for k in _HEADER_FLOAT:
            setattr(self, k, float(fields.get(k, 0.0)))
        self.rawdatafile = str(fields.get("rawdatafile", ""))
        self.source_name = str(fields.get("source_name", ""))
        self.frequency_table = [float(f) for f in (frequency_table if frequency_table is not None else [])]
        self.uses_frequency_table = bool(fields.get("uses_frequency_table", False))

    def __repr__(self) -> str:
        return (f"FilterbankHeader(nsamples={self.nsamples}, nchans={self.nchans}, nifs={self.nifs}, "
                f"nbits={self.nbits}, tsamp={self.tsamp}, fch1={self.fch1}, foff={self.foff})")


class Filterbank:
    """In-memory SIGPROC filterbank, data (nsamples, nifs, nchans); channels in
    ascending frequency unless channel_order="preserve_file_order"
    (filterbank_bindings.cpp, io/filterbank.cpp:116-348).  The file is read
    by the library's reader (gf_filterbank_read_host)."""

    def __init__(self, path, *, channel_order: str = "frequency_ascending", reverse_backend: str = "auto",
                 io_buffer_bytes: int = 67_108_864, openmp_min_rows: int = 4096):
        if channel_order not in ("frequency_ascending", "preserve_file_order"):
            raise ValueError(f"unknown channel_order: {channel_order}")
        if reverse_backend not in ("auto", "cpu_scalar", "cpu_openmp"):
            raise ValueError(f"unknown reverse_backend: {reverse_backend}")
        if io_buffer_bytes <= 0:
            raise ValueError("io_buffer_bytes must be positive")
        h, freq, data = core.read_filterbank(Path(path), preserve_file_order=channel_order == "preserve_file_order")
        self.header = FilterbankHeader(h, freq)
        self.data = data

    @property
    def shape(self) -> tuple:
        return tuple(self.data.shape)

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def nbytes(self) -> int:
        return int(self.data.nbytes)

    def __repr__(self) -> str:
        return f"Filterbank(shape={self.shape}, dtype={self.dtype})"


# ---------------------------------------------------------------------------
# result wrappers (dedispersion_bindings.cpp:75-185)
# ---------------------------------------------------------------------------

def _require_array(data, name: str) -> np.ndarray:
    if not isinstance(data, np.ndarray):
        raise TypeError(f"{name} must be a numpy.ndarray")
    if data.ndim != 2:
        raise ValueError(f"{name} must be a 2D array")
    if data.size == 0:
        raise ValueError(f"{name} must not be empty")
    if not data.flags.c_contiguous:
        raise ValueError(f"{name} must be C-contiguous; use numpy.ascontiguousarray explicitly if a copy is "
                         "intended")
    return data


def _finite_nonneg(value: float, name: str) -> float:
    value = float(value)
    if not (math.isfinite(value) and value >= 0.0):
        raise ValueError(f"{name} must be finite and non-negative")
    return value


def _tsamp(value: float) -> float:
    value = float(value)
    if not (math.isfinite(value) and value > 0.0):
        raise ValueError("tsamp must be finite and positive")
    return value


class DedispersedResult:
    """Host-resident dedispersed series, data (ndm, nsamples) uint32 or float32,
    wrapped without a copy."""

    def __init__(self, data, *, tsamp: float, dm_low: float = 0.0, dm_step: float = 0.0,
                 backend: str = "external"):
        data = _require_array(data, "dedispersed result data")
        if data.dtype not in (np.uint32, np.float32):
            raise TypeError("dedispersed result data must have dtype uint32 or float32")
        self.data = data
        self.tsamp = _tsamp(tsamp)
        self.dm_low = _finite_nonneg(dm_low, "dm_low")
        self.dm_step = _finite_nonneg(dm_step, "dm_step")
        self.backend = str(backend)

    ndm = property(lambda self: int(self.data.shape[0]))
    nsamples = property(lambda self: int(self.data.shape[1]))
    shape = property(lambda self: tuple(self.data.shape))
    dtype = property(lambda self: self.data.dtype)
    nbytes = property(lambda self: int(self.data.nbytes))

    def __repr__(self) -> str:
        return (f"DedispersedResult(ndm={self.ndm}, nsamples={self.nsamples}, dtype={self.dtype}, "
                f"backend={self.backend!r})")


class DedispersedSpectrum:
    """Host-resident aligned dynamic spectrum, data (nsamples, nchans) uint8,
    uint16 or float32, wrapped without a copy."""

    def __init__(self, data, *, tsamp: float, dm: float = 0.0, chan_begin: int = 0, chan_end: int | None = None,
                 backend: str = "external"):
        data = _require_array(data, "dedispersed spectrum data")
        if data.dtype not in (np.uint8, np.uint16, np.float32):
            raise TypeError("dedispersed spectrum data must have dtype uint8, uint16 or float32")
        self.data = data
        self.tsamp = _tsamp(tsamp)
        self.dm = _finite_nonneg(dm, "dm")
        if chan_begin < 0:
            raise ValueError("chan_begin must be non-negative")
        end = chan_begin + data.shape[1] if chan_end is None else chan_end
        if end < 0:
            raise ValueError("chan_end must be non-negative")
        if end - chan_begin != data.shape[1]:
            raise ValueError("chan_end - chan_begin must equal data.shape[1]")
        self.chan_begin, self.chan_end = int(chan_begin), int(end)
        self.backend = str(backend)

    nsamples = property(lambda self: int(self.data.shape[0]))
    nchans = property(lambda self: int(self.data.shape[1]))
    shape = property(lambda self: tuple(self.data.shape))
    dtype = property(lambda self: self.data.dtype)
    nbytes = property(lambda self: int(self.data.nbytes))

    def __repr__(self) -> str:
        return f"DedispersedSpectrum(dm={self.dm}, shape={self.shape}, dtype={self.dtype}, backend={self.backend!r})"


# ---------------------------------------------------------------------------
# dedispersion (dedispersion_bindings.cpp:648-672)
# ---------------------------------------------------------------------------

def _filterbank_samples(filterbank: Filterbank) -> tuple[np.ndarray, np.ndarray, float]:
    """validate_filterbank_header + typed_sample_view
    (dedispersion_bindings.cpp:194-257): (time-major [nsamples][nchans]
    samples, frequencies, tsamp)."""
    h = filterbank.header
    if h.nsamples <= 0:
        raise ValueError("dedispersion requires at least one sample")
    if h.nifs != 1:
        raise ValueError("dedispersion requires nifs == 1")
    if h.nchans <= 0:
        raise ValueError("dedispersion requires at least one channel")
    if not h.tsamp > 0.0:
        raise ValueError("filterbank tsamp must be positive")
    if len(h.frequency_table) != h.nchans:
        raise ValueError("filterbank frequency table length must match nchans")
    data = filterbank.data
    if not isinstance(data, np.ndarray) or data.ndim != 3:
        raise ValueError("filterbank data must be a 3D numpy array")
    if data.shape != (h.nsamples, h.nifs, h.nchans):
        raise ValueError("filterbank data shape does not match header")
    if not data.flags.c_contiguous:
        raise ValueError("filterbank data must be C-contiguous in (time, if, channel) order")
    return data.reshape(h.nsamples, h.nchans), np.asarray(h.frequency_table, np.float64), float(h.tsamp)


def _require_u8(samples: np.ndarray) -> None:
    if samples.dtype != np.uint8:
        if samples.dtype in (np.uint16, np.float32):
            raise TypeError("gaffa_b200 dedisperses 8-bit filterbanks; 16-bit and float32 samples are "
                            "taken by dedisperse_spectrum only")
        raise TypeError("unsupported filterbank sample dtype")


def _dedisperse(filterbank: Filterbank, dm_low: float, dm_step: float, ndm: int, algorithm: str,
                subband_channels: int, ndm_per_nominal: int, device_id: int, backend: str,
                threads_per_block: int, time_tile_samples: int) -> DedispersedResult:
    import torch
    _backend(backend)
    dev = _device(device_id)
    if threads_per_block <= 0 or time_tile_samples <= 0:
        raise ValueError("threads_per_block and time_tile_samples must be positive")
    dm_low = _finite_nonneg(dm_low, "dm_low")
    dm_step = _finite_nonneg(dm_step, "dm_step")
    if ndm <= 0:
        raise ValueError("ndm must be positive")
    samples, freq, tsamp = _filterbank_samples(filterbank)
    _require_u8(samples)
    # a one-DM grid has no spacing; the program takes any positive step for it
    prog_step = dm_step if ndm > 1 else (dm_step or 1.0)
    prog = core.DedispersionProgram(freq, samples.shape[0], tsamp, dm_low, prog_step, int(ndm), nbits=8,
                                    algorithm=algorithm, subband_channels=subband_channels,
                                    ndm_per_nominal=ndm_per_nominal, device_id=dev)
    with torch.cuda.device(dev):
        staged = prog.stage(torch.from_numpy(np.ascontiguousarray(samples)).to(f"cuda:{dev}"))
        out = prog.run(staged, 0, int(ndm))
        prog.check()
        host = out[:, : prog.nout].contiguous().cpu().numpy().view(np.uint32)
    return DedispersedResult(np.ascontiguousarray(host), tsamp=tsamp, dm_low=dm_low,
                             dm_step=dm_step if ndm > 1 or algorithm == "subband" else 0.0, backend="cuda")


def dedisperse_spectrum(filterbank: Filterbank, *, dm: float, backend: str = "cuda", device_id: int = 0,
                        threads_per_block: int = 256, time_tile_samples: int = 81920) -> DedispersedSpectrum:
    """Aligned single-DM dynamic spectrum (dedisperse_spectrum_cuda,
    dedispersion_cuda.cu:295-318); input dtype preserved."""
    import torch
    _backend(backend)
    dev = _device(device_id)
    dm = _finite_nonneg(dm, "dm")
    samples, freq, tsamp = _filterbank_samples(filterbank)
    if samples.dtype not in (np.uint8, np.uint16, np.float32):
        raise TypeError("unsupported filterbank sample dtype")
    src = samples.view(np.int16) if samples.dtype == np.uint16 else samples
    with torch.cuda.device(dev):
        out = core.dedisperse_spectrum(torch.from_numpy(np.ascontiguousarray(src)).to(f"cuda:{dev}"), freq, dm,
                                       tsamp)
        host = out.cpu().numpy()
    if samples.dtype == np.uint16:
        host = host.view(np.uint16)
    return DedispersedSpectrum(np.ascontiguousarray(host), tsamp=tsamp, dm=dm, backend="cuda")


def dedisperse_single_dm(filterbank: Filterbank, *, dm: float, backend: str = "cuda", device_id: int = 0,
                         threads_per_block: int = 256, time_tile_samples: int = 81920) -> DedispersedResult:
    """One DM (dedisperse_single_dm_cuda): data (1, nsamples - delay(dm))."""
    return _dedisperse(filterbank, dm, 0.0, 1, "brute", 32, 32, device_id, backend, threads_per_block,
                       time_tile_samples)


def dedisperse_multi_dm(filterbank: Filterbank, *, dm_low: float, dm_step: float, ndm: int, backend: str = "cuda",
                        device_id: int = 0, threads_per_block: int = 256,
                        time_tile_samples: int = 81920) -> DedispersedResult:
    """Contiguous DM grid by direct sums (dedisperse_multi_dm_cuda): row i is
    dm_low + i * dm_step; all rows share the valid-only length."""
    return _dedisperse(filterbank, dm_low, dm_step, ndm, "brute", 32, 32, device_id, backend, threads_per_block,
                       time_tile_samples)


def dedisperse_subband(filterbank: Filterbank, *, dm_low: float, dm_step: float, ndm: int, backend: str = "cuda",
                       subband_channels: int = 32, ndm_per_nominal: int = 32, device_id: int = 0,
                       threads_per_block: int = 256, time_tile_samples: int = 81920) -> DedispersedResult:
    """Two-stage subband dedispersion (dedisperse_subband_cuda,
    dedispersion.cpp:331-453 arithmetic)."""
    if subband_channels <= 0 or ndm_per_nominal <= 0:
        raise ValueError("subband_channels and ndm_per_nominal must be positive")
    return _dedisperse(filterbank, dm_low, dm_step, ndm, "subband", int(subband_channels), int(ndm_per_nominal),
                       device_id, backend, threads_per_block, time_tile_samples)


# ---------------------------------------------------------------------------
# FFA (ffa_bindings.cpp:160-217)
# ---------------------------------------------------------------------------

class FfaPlan:
    """Immutable FFA search plan (FfaSearchPlan, include/gaffa/ffa_plan.h:49-53)."""

    def __init__(self, plan: core.FfaPlan, nsamples: int):
        self._plan = plan
        self._nsamples = int(nsamples)

    @property
    def task_count(self) -> int:
        return self._plan.task_count

    @property
    def width_trials(self) -> tuple:
        return self._plan.width_trials

    def __repr__(self) -> str:
        return f"FfaPlan(task_count={self.task_count}, width_trials={self.width_trials})"


class FfaPeak:
    """One raw FFA peak (FfaPeak, include/gaffa/ffa_peak.h:8-19)."""

    __slots__ = ("period", "frequency", "snr", "width", "duty_cycle", "phase", "shift", "bins", "width_index",
                 "period_index")

    def __init__(self, rec):
        self.period = float(rec["period"])
        self.frequency = float(rec["frequency"])
        self.snr = float(rec["snr"])
        self.width = int(rec["width"])
        self.duty_cycle = float(rec["duty_cycle"])
        self.phase = int(rec["phase"])
        self.shift = int(rec["shift"])
        self.bins = int(rec["bins"])
        self.width_index = int(rec["width_index"])
        self.period_index = int(rec["period_index"])

    def __repr__(self) -> str:
        return (f"FfaPeak(period={self.period}, snr={self.snr}, width={self.width}, phase={self.phase}, "
                f"bins={self.bins})")


def _make_riptide_ffa_plan(*, nsamples: int, tsamp: float, period_min: float, period_max: float,
                           bins_min: int = 180, bins_max: int = 256, min_periods: int = 1,
                           duty_cycle_max: float = 0.20, width_trial_spacing: float = 1.5,
                           max_tasks: int = 1_000_000) -> FfaPlan:
    """make_riptide_ffa_plan (ffa_plan.cpp:90-170)."""
    plan = core.make_riptide_ffa_plan(int(nsamples), float(tsamp), float(period_min), float(period_max),
                                      bins_min=int(bins_min), bins_max=int(bins_max), min_periods=int(min_periods),
                                      duty_cycle_max=float(duty_cycle_max),
                                      width_trial_spacing=float(width_trial_spacing), max_tasks=int(max_tasks))
    return FfaPlan(plan, nsamples)


def _validate_series(time_series) -> np.ndarray:
    """validate_time_series_array (ffa_bindings.cpp:54-70)."""
    if not isinstance(time_series, np.ndarray):
        raise TypeError("FFA time_series must be a numpy.ndarray")
    if time_series.ndim != 1:
        raise ValueError("FFA time_series must be a 1D array")
    if time_series.shape[0] <= 0:
        raise ValueError("FFA time_series must not be empty")
    if time_series.dtype != np.float32:
        raise TypeError("FFA time_series must have dtype float32")
    if time_series.strides[0] != 4:
        raise ValueError("FFA time_series must be C-contiguous; use numpy.ascontiguousarray explicitly if a copy "
                         "is intended")
    return time_series


def _peak_limit(max_peaks) -> int:
    if max_peaks is None:
        return 0
    limit = int(max_peaks)
    if limit <= 0:
        raise ValueError("max_peaks must be positive or None")
    return limit


def _ffa_search_cpu(time_series, plan: FfaPlan, *, snr_threshold: float = 6.0, max_peaks=None):
    """Not provided: this library has no CPU path."""
    raise ValueError(CPU_BACKEND_MESSAGE)


def _ffa_search_cuda_host(time_series, plan: FfaPlan, *, device_id: int = 0, snr_threshold: float = 6.0,
                          max_peaks=None) -> list:
    """search_ffa_cuda of one host float32 series (ffa_bindings.cpp:120-158):
    uploads it, searches every task of the plan, returns the raw peaks in
    the reference's deterministic order (is_better_ffa_peak)."""
    import torch
    x = _validate_series(time_series)
    limit = _peak_limit(max_peaks)
    dev = _device(device_id)
    thr = float(snr_threshold)
    if not math.isfinite(thr):
        raise ValueError("FFA search S/N threshold must be finite")
    if x.shape[0] != plan._plan.nsamples:
        raise ValueError("FFA executor task input_nsamples must match time series size")
    with torch.cuda.device(dev):
        prog = core.FfaProgram(plan._plan, max_series=1, device_id=dev)
        s = torch.from_numpy(x).to(f"cuda:{dev}").view(1, -1)
        prep = prog.prepare(s, 1)
        rec = prog.search(prep, 1, thr, max_peaks=limit)
        peaks = core.sort_peaks(prog.expand(rec))
    return [FfaPeak(p) for p in peaks]


# ---------------------------------------------------------------------------
# folding (folding_bindings.cpp)
# ---------------------------------------------------------------------------

class FoldedProfile:
    """Integrated profile of a folded series (FoldedProfile, folding.h)."""

    def __init__(self, profile, exposure, nbin, period, tsamp):
        self.profile = np.asarray(profile, np.float32)
        self.exposure = np.asarray(exposure, np.float64)
        self.nbin = int(nbin)
        self.period = float(period)
        self.tsamp = float(tsamp)
        self.phase = (np.arange(self.nbin, dtype=np.float64) / self.nbin).astype(np.float32)

    def __repr__(self) -> str:
        return f"FoldedProfile(nbin={self.nbin}, period={self.period})"


class FoldResult:
    """Folded spectrum products (FoldResult, folding.h): cube (nsubint, nchans,
    nbin), exposure (nsubint, nbin), profile, freq_phase, time_phase."""

    def __init__(self, products: dict, period: float, tsamp: float):
        self.cube = products["cube"].cpu().numpy()
        self.exposure = products["exposure"].cpu().numpy()
        self.profile = products["profile"].cpu().numpy()
        self.freq_phase = products["freq_phase"].cpu().numpy()
        self.time_phase = products["time_phase"].cpu().numpy()
        self.nsubint, self.nchans, self.nbin = (int(v) for v in self.cube.shape)
        self.period = float(period)
        self.tsamp = float(tsamp)
        self.tsubint = float(products["tsubint"])
        self.phase = (np.arange(self.nbin, dtype=np.float64) / self.nbin).astype(np.float32)
        self.time = (np.arange(self.nsubint, dtype=np.float64) + 0.5) * self.tsubint  # subint centres

    def __repr__(self) -> str:
        return f"FoldResult(nsubint={self.nsubint}, nchans={self.nchans}, nbin={self.nbin}, period={self.period})"


def _fold_args(period: float, nbin: int) -> None:
    if not (math.isfinite(float(period)) and float(period) > 0.0):
        raise ValueError("fold period must be finite and positive")
    if int(nbin) <= 0:
        raise ValueError("fold nbin must be positive")


def _fold_dedispersed_profile(data, *, tsamp: float, period: float, nbin: int, dm_index: int = 0,
                              device_id: int = 0) -> FoldedProfile:
    """fold_time_series of one row of a dedispersed array
    (folding_bindings.cpp:95-135, folding.cpp:452-502)."""
    import torch
    data = _require_array(data, "dedispersed result data")
    if data.dtype not in (np.uint32, np.float32):
        raise TypeError("dedispersed result data dtype mismatch")
    if not 0 <= int(dm_index) < data.shape[0]:
        raise IndexError("dm_index is out of range")
    tsamp = _tsamp(tsamp)
    _fold_args(period, nbin)
    row = np.ascontiguousarray(data[int(dm_index)])
    if row.dtype == np.uint32:
        row = row.view(np.int32)
    dev = _device(device_id)
    with torch.cuda.device(dev):
        prof, expo = core.fold_time_series(torch.from_numpy(row).to(f"cuda:{dev}"), float(period), tsamp,
                                           int(nbin))
    return FoldedProfile(prof, expo, nbin, period, tsamp)


def _fold_dedispersed_spectrum(data, *, tsamp: float, period: float, nbin: int, tsubint: float,
                               output_channels: int, device_id: int = 0) -> FoldResult:
    """fold_dedispersed_spectrum of an aligned spectrum
    (folding_bindings.cpp:137-160, folding.cpp:408-438)."""
    import torch
    data = _require_array(data, "dedispersed spectrum data")
    if data.dtype not in (np.uint8, np.uint16, np.float32):
        raise TypeError("dedispersed spectrum data dtype mismatch")
    tsamp = _tsamp(tsamp)
    _fold_args(period, nbin)
    if not (math.isfinite(float(tsubint)) and float(tsubint) > 0.0):
        raise ValueError("fold tsubint must be finite and positive")
    if output_channels < 0:
        raise ValueError("output_channels must be non-negative")
    if output_channels and data.shape[1] % output_channels:
        raise ValueError("output_channels must divide the channel count")
    src = data.view(np.int16) if data.dtype == np.uint16 else data
    dev = _device(device_id)
    with torch.cuda.device(dev):
        spec = torch.from_numpy(np.ascontiguousarray(src)).to(f"cuda:{dev}")
        sub = max(1, int(round(float(tsubint) / tsamp)))
        cube, expo = core.fold_spectrum(spec, float(period), tsamp, int(nbin), sub, 0, int(output_channels))
        products = _project(cube, expo)
        products["tsubint"] = sub * tsamp
    return FoldResult(products, period, tsamp)


def _project(cube, expo) -> dict:
    import ctypes as C

    import torch
    nsub, nch, nbin = cube.shape
    prof = torch.empty(nbin, dtype=torch.float32, device=cube.device)
    fp = torch.empty((nch, nbin), dtype=torch.float32, device=cube.device)
    tp = torch.empty((nsub, nbin), dtype=torch.float32, device=cube.device)
    s = torch.cuda.current_stream(cube.device)
    _lib.check(_lib.lib().gf_project_folded_cube(_lib.ptr(cube), _lib.ptr(expo), nsub, nch, nbin, _lib.ptr(prof),
                                                 _lib.ptr(fp), _lib.ptr(tp), C.c_void_p(s.cuda_stream)))
    return {"cube": cube, "exposure": expo, "profile": prof, "freq_phase": fp, "time_phase": tp}
