"""Device programs over the C ABI (include/gaffa_b200.h).

Each class owns the library's program handle (device metadata) and allocates
its work buffers with torch on the program's device; torch is only the
allocator and stream provider here -- every computation is a gf_* call into
libgaffa_b200.so.  All calls are stream-ordered on the current torch stream
and never synchronise implicitly, except where a host result is returned.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr


def _stream(stream=None):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _require_cuda(device_id: int) -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("gaffa_b200 needs a CUDA device (no CPU fallback)")
    if device_id < 0 or device_id >= torch.cuda.device_count():
        raise ValueError(f"device_id {device_id} out of range")
    return torch.device("cuda", device_id)


# ---------------------------------------------------------------------------
# FFA plan (host)
# ---------------------------------------------------------------------------

class FfaPlan:
    """Riptide FFA plan: tasks (TASK_DTYPE records) and width trials.

    Mirrors gaffa's FfaPlan / FfaSearchPlan (include/gaffa/ffa_plan.h); the
    width trials may be replaced as FfaSearchPlan::width_trials allows.
    """

    def __init__(self, tasks: np.ndarray, width_trials):
        self.tasks = np.ascontiguousarray(tasks, _lib.TASK_DTYPE)
        self.width_trials = tuple(int(w) for w in width_trials)

    @property
    def task_count(self) -> int:
        return len(self.tasks)

    @property
    def nsamples(self) -> int:
        return int(self.tasks[0]["input_nsamples"]) if len(self.tasks) else 0

    @property
    def prepared_floats(self) -> int:
        """Floats of one prepared series: every distinct downsample factor's
        samples, each rounded up to 4 (the FFA program's layout), known
        before any program exists."""
        seen, off = set(), 0
        for t in self.tasks:
            f = float(t["downsample_factor"])
            if f not in seen:
                seen.add(f)
                off = (off + int(t["prepared_nsamples"]) + 3) // 4 * 4
        return off

    def with_widths(self, widths) -> "FfaPlan":
        return FfaPlan(self.tasks, widths)

    def __repr__(self):
        return f"FfaPlan(task_count={self.task_count}, width_trials={self.width_trials})"


def make_riptide_ffa_plan(nsamples: int, tsamp: float, period_min: float, period_max: float,
                          bins_min: int = 180, bins_max: int = 256, min_periods: int = 1,
                          duty_cycle_max: float = 0.20, width_trial_spacing: float = 1.5,
                          max_tasks: int = 1_000_000) -> FfaPlan:
    """make_riptide_ffa_plan (src/gaffa/ffa_plan.cpp:90-170) via gf_make_riptide_ffa_plan."""
    L = _lib.lib()
    o = _lib.PlanOptions(period_min, period_max, bins_min, bins_max, min_periods, duty_cycle_max,
                         width_trial_spacing, max_tasks)
    nt, nw = _lib.u64(), _lib.u64()
    check(L.gf_make_riptide_ffa_plan(nsamples, tsamp, C.byref(o), None, 0, C.byref(nt), None, 0, C.byref(nw)))
    tasks = np.zeros(nt.value, _lib.TASK_DTYPE)
    widths = np.zeros(nw.value, np.uint64)
    check(L.gf_make_riptide_ffa_plan(nsamples, tsamp, C.byref(o), ptr(tasks), len(tasks), C.byref(nt),
                                     ptr(widths), len(widths), C.byref(nw)))
    return FfaPlan(tasks, widths)


# ---------------------------------------------------------------------------
# dedispersion
# ---------------------------------------------------------------------------

class DedispersionProgram:
    """Delay tables and gather records for one observation geometry.

    Counterpart of the host set-up inside dedisperse_*_cuda_device
    (src/gaffa/dedispersion_cuda.cu:536-714).
    """

    def __init__(self, frequency_mhz, nsamples: int, tsamp: float, dm_low: float, dm_step: float,
                 ndm: int, ref_frequency_mhz: float | None = None, chan_begin: int = 0,
                 chan_end: int | None = None, nbits: int = 8, algorithm: str = "brute",
                 subband_channels: int = 32, ndm_per_nominal: int = 32, device_id: int = 0,
                 launch_shape: tuple[int, int] | None = None):
        self.device = _require_cuda(device_id)
        self.device_id = device_id
        self.launch_shape = launch_shape
        self.freq = np.ascontiguousarray(frequency_mhz, np.float64)
        nchans = len(self.freq)
        self.nbits = nbits
        self.nchans = nchans
        self.nsamples = nsamples
        self.ndm = ndm
        self.algorithm = algorithm
        self.ndm_per_nominal = ndm_per_nominal
        fref = float(self.freq.max()) if ref_frequency_mhz is None else float(ref_frequency_mhz)
        d = _lib.DedispDesc()
        d.nsamples, d.nchans = nsamples, nchans
        d.frequency_mhz = self.freq.ctypes.data_as(C.POINTER(C.c_double))
        d.dm_low, d.dm_step, d.ndm = dm_low, dm_step, ndm
        d.ref_frequency_mhz, d.tsamp = fref, tsamp
        d.chan_begin = chan_begin
        d.chan_end = nchans if chan_end is None else chan_end
        d.nbits = nbits
        d.algorithm = {"brute": _lib.DEDISP_BRUTE, "subband": _lib.DEDISP_SUBBAND}[algorithm]
        d.subband_channels, d.ndm_per_nominal = subband_channels, ndm_per_nominal
        d.device_id = device_id
        if launch_shape is not None:
            # (DMs per CTA, channel rows per staging step); 0 = automatic
            d.launch_dms_per_cta, d.launch_chunk_rows = launch_shape
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_dedisp_program_create(C.byref(d), C.byref(h)))
        self._h = h
        info = _lib.DedispInfo()
        check(_lib.lib().gf_dedisp_program_info(h, C.byref(info)))
        self.info = info
        self.nout = int(info.nout)
        self.dm_low, self.dm_step, self.tsamp = dm_low, dm_step, tsamp

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.gf_dedisp_program_destroy(h)

    __del__ = close

    @property
    def row_bytes(self) -> int:
        return self.nchans if self.nbits == 8 else self.nchans // 4

    @property
    def batch_granularity(self) -> int:
        return 8 if self.algorithm == "brute" else self.ndm_per_nominal

    def workspace_bytes(self, dm_count: int) -> int:
        b = _lib.u64()
        check(_lib.lib().gf_dedisp_workspace_bytes(self._h, dm_count, C.byref(b)))
        return int(b.value)

    def stage(self, data, stream=None, out: torch.Tensor | None = None) -> torch.Tensor:
        """Channel-major staging of a time-major input (device tensor, or host
        numpy array / tensor copied through a bounce buffer), into `out` when
        given (uint8, at least staged_bytes)."""
        if out is None:
            staged = torch.empty(int(self.info.staged_bytes), dtype=torch.uint8, device=self.device)
        else:
            if out.dtype != torch.uint8 or out.numel() < self.info.staged_bytes or out.device != self.device:
                raise ValueError("staging buffer must be uint8 on the program's device with staged_bytes bytes")
            staged = out
        with torch.cuda.device(self.device):
            if isinstance(data, torch.Tensor) and data.is_cuda:
                if data.numel() * data.element_size() != self.info.input_bytes:
                    raise ValueError("input size does not match the program geometry")
                check(_lib.lib().gf_dedisp_stage(self._h, ptr(data), ptr(staged), _stream(stream)))
            else:
                host = data if isinstance(data, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(data))
                if host.numel() * host.element_size() != self.info.input_bytes:
                    raise ValueError("input size does not match the program geometry")
                bounce_rows = max(128, (256 << 20) // self.row_bytes)
                bounce = torch.empty(2 * bounce_rows * self.row_bytes, dtype=torch.uint8, device=self.device)
                if not host.is_pinned():
                    host = host.pin_memory()
                check(_lib.lib().gf_dedisp_stage_from_host(self._h, ptr(host), ptr(staged), ptr(bounce),
                                                           bounce.numel(), _stream(stream)))
                torch.cuda.current_stream().synchronize()
        return staged

    def run(self, staged: torch.Tensor, dm_begin: int = 0, dm_count: int | None = None,
            out: torch.Tensor | None = None, out_stride: int | None = None,
            workspace: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        """Dedisperse DMs [dm_begin, dm_begin + dm_count) into uint32
        [dm_count][out_stride] (a view of `out` when given)."""
        dm_count = self.ndm - dm_begin if dm_count is None else dm_count
        out_stride = out_stride or ((self.nout + 3) // 4) * 4
        if out is None:
            out = torch.empty(dm_count * out_stride, dtype=torch.int32, device=self.device)
        if self.algorithm == "subband" and workspace is None:
            workspace = torch.empty(self.workspace_bytes(dm_count), dtype=torch.uint8, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_dedisp_run(self._h, ptr(staged), dm_begin, dm_count, ptr(out), out_stride,
                                           ptr(workspace), _stream(stream)))
        return out.view(-1)[: dm_count * out_stride].view(dm_count, out_stride)

    def check(self, stream=None) -> None:
        """Synchronises the stream and raises if a launch of this program gave
        up waiting for a shared-memory copy stage (gf_dedisp_check)."""
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_dedisp_check(self._h, _stream(stream)))


class DedispersionBatch:
    """Many brute-force (program, staged input, DM range, output) items of
    different observations as one kernel launch (gf_dedisp_batch_*).  Device
    pointers are fixed here, so run() can be captured in a CUDA graph; the
    tensors must stay alive as long as the batch."""

    def __init__(self, items):
        items = list(items)
        if not items:
            raise ValueError("batched dedispersion needs at least one item")
        arr = (_lib.DedispBatchItem * len(items))()
        self._keep = []
        device = None
        for i, (program, staged, dm_begin, dm_count, out, out_stride) in enumerate(items):
            if program.algorithm != "brute":
                raise ValueError("batched dedispersion takes brute-force programs")
            if out.numel() < dm_count * out_stride:
                raise ValueError("output too small for the DM range")
            arr[i].program = program._h
            arr[i].dev_staged = ptr(staged)
            arr[i].dm_begin, arr[i].dm_count = dm_begin, dm_count
            arr[i].dev_out = ptr(out)
            arr[i].out_stride = out_stride
            self._keep += [program, staged, out]
            device = program.device
        self.device = device
        h = C.c_void_p()
        with torch.cuda.device(device):
            check(_lib.lib().gf_dedisp_batch_create(arr, len(items), C.byref(h)))
        self._h = h

    def run(self, stream=None) -> None:
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_dedisp_batch_run(self._h, _stream(stream)))

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.gf_dedisp_batch_destroy(h)

    __del__ = close


# ---------------------------------------------------------------------------
# preprocessing
# ---------------------------------------------------------------------------

class PreprocessProgram:
    """Riptide running-median detrend + normalise (CudaPreprocessProgram of
    include/gaffa/preprocessing_cuda.h:44-89) for series of one length."""

    def __init__(self, nsamples: int, tsamp: float, window_seconds: float = 5.0, min_points: int = 101,
                 normalise: bool = True, reject_constant: bool = True, max_series: int = 16,
                 device_id: int = 0):
        self.device = _require_cuda(device_id)
        self.desc = _lib.PreprocessDesc(tsamp, window_seconds, min_points, int(normalise),
                                        int(reject_constant), nsamples, max_series)
        self.info = _lib.PreprocessInfo()
        check(_lib.lib().gf_preprocess_info_get(C.byref(self.desc), C.byref(self.info)))
        self.workspace = torch.empty(max(16, int(self.info.workspace_bytes)), dtype=torch.uint8,
                                     device=self.device)
        self.stats = torch.zeros((max_series, 2), dtype=torch.float64, device=self.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.nsamples = nsamples
        self.max_series = max_series
        self.normalise = normalise

    def run(self, series: torch.Tensor, nseries: int | None = None, stream=None) -> torch.Tensor:
        """In place on [nseries][stride] uint32 (int32 storage) or float32.
        Returns the [nseries][2] FP64 (mean, 1/stddev) table."""
        if series.dim() != 2:
            raise ValueError("series must be [nseries][stride]")
        nseries = series.shape[0] if nseries is None else nseries
        is_u32 = series.dtype in (torch.int32, torch.uint32)
        if not is_u32 and series.dtype != torch.float32:
            raise TypeError("series must be uint32 (int32 storage) or float32")
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_preprocess_inplace(C.byref(self.desc), ptr(series), int(is_u32), nseries,
                                                   series.stride(0), ptr(self.workspace), ptr(self.stats),
                                                   ptr(self.status), _stream(stream)))
        return self.stats[:nseries]

    def synchronize(self) -> None:
        """Waits and raises the deferred data error, as
        CudaPreprocessProgram::synchronize (preprocessing_cuda.cu:781-817)."""
        torch.cuda.current_stream(self.device).synchronize()
        st = int(self.status.item())
        self.status.zero_()
        if st & _lib.STATUS_NONFINITE:
            raise ValueError("running median detrend input samples must be finite")
        if st & _lib.STATUS_CONSTANT:
            raise ValueError("normalise input standard deviation must be finite and > 0")

    def normalise_inplace(self, series: torch.Tensor, nseries: int, stream=None) -> None:
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_normalise(ptr(series), nseries, series.stride(0), self.nsamples,
                                          ptr(self.stats), _stream(stream)))


class PreprocessBatch:
    """Many PreprocessProgram.run calls (series sets of different lengths and
    windows) as one launch per stage (gf_preprocess_batch_*).  items:
    [(PreprocessProgram, series [nseries][stride] int32 or float32, nseries)];
    each program's statistics and status receive its item's results, as
    run() would.  Pointers are fixed here, so run() can be captured in a CUDA
    graph; the tensors must stay alive as long as the batch."""

    def __init__(self, items):
        items = list(items)
        if not items:
            raise ValueError("batched preprocessing needs at least one item")
        arr = (_lib.PreprocessBatchItem * len(items))()
        self._keep = []
        device = None
        for i, (pre, series, nseries) in enumerate(items):
            if series.dim() != 2:
                raise ValueError("series must be [nseries][stride]")
            is_u32 = series.dtype in (torch.int32, torch.uint32)
            if not is_u32 and series.dtype != torch.float32:
                raise TypeError("series must be uint32 (int32 storage) or float32")
            arr[i].desc = C.pointer(pre.desc)
            arr[i].dev_series = ptr(series)
            arr[i].input_is_u32 = int(is_u32)
            arr[i].nseries, arr[i].stride = int(nseries), series.stride(0)
            arr[i].dev_workspace, arr[i].dev_stats, arr[i].dev_status = ptr(pre.workspace), ptr(pre.stats), \
                ptr(pre.status)
            self._keep += [pre, series]
            if device is not None and pre.device != device:
                raise ValueError("batched preprocessing items must share one device")
            device = pre.device
        self.device = device
        h = C.c_void_p()
        with torch.cuda.device(device):
            check(_lib.lib().gf_preprocess_batch_create(arr, len(items), device.index or 0, C.byref(h)))
        self._h = h
        self.scrunched = any(int(p.info.scrunch_factor) > 1 for p, _, _ in items)

    @property
    def kernel_launches(self) -> int:
        return 4 if self.scrunched else 3

    def run(self, stream=None) -> None:
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_preprocess_batch_run(self._h, _stream(stream)))

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.gf_preprocess_batch_destroy(h)

    __del__ = close


# ---------------------------------------------------------------------------
# FFA
# ---------------------------------------------------------------------------

class FfaProgram:
    """Device tables for one FFA plan (CudaFfaProgram,
    src/gaffa/ffa_cuda_executor.cuh:44-80)."""

    def __init__(self, plan: FfaPlan, max_series: int = 16, device_id: int = 0):
        self.device = _require_cuda(device_id)
        self.plan = plan
        self.max_series = max_series
        widths = np.ascontiguousarray(plan.width_trials, np.uint64)
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_program_create(ptr(plan.tasks), len(plan.tasks), ptr(widths), len(widths),
                                                   max_series, device_id, C.byref(h)))
        self._h = h
        self.info = _lib.FfaInfo()
        check(_lib.lib().gf_ffa_program_info(h, C.byref(self.info)))
        self.scratch = torch.empty(max(16, int(self.info.scratch_bytes)), dtype=torch.uint8, device=self.device)
        self.counters = torch.zeros(2, dtype=torch.int64, device=self.device)
        self.capacity = 1 << 16
        self.peaks = torch.empty(self.capacity * 24, dtype=torch.uint8, device=self.device)

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.gf_ffa_program_destroy(h)

    __del__ = close

    @property
    def prepared_floats(self) -> int:
        return int(self.info.prepared_floats)

    def prepare(self, series: torch.Tensor, nseries: int, stats: torch.Tensor | None = None,
                out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        if out is None:
            out = torch.empty((nseries, self.prepared_floats), dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_prepare(self._h, ptr(series), nseries, series.stride(0), ptr(stats), ptr(out),
                                            _stream(stream)))
        return out

    def search_async(self, prepared: torch.Tensor, nseries: int, snr_threshold: float, stream=None):
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_search(self._h, ptr(prepared), nseries, snr_threshold, ptr(self.scratch),
                                           ptr(self.peaks), self.capacity, ptr(self.counters), _stream(stream)))

    @property
    def kernel_launches(self) -> int:
        return int(self.info.nclasses)

    def count(self, prepared: torch.Tensor, nseries: int, snr_threshold: float, max_peaks: int = 0,
              stream=None) -> int:
        """Peak records of the last search_async, left on the device in
        self.peaks (the first count * 24 bytes); grows the buffer and re-runs
        on overflow as collect does."""
        while True:
            counts = self.counters.cpu()
            if int(counts[1]) & _lib.STATUS_SCHEDULE:
                raise RuntimeError("FFA block schedule exceeded its shared-memory tile")
            n = int(counts[0])
            if n <= self.capacity:
                break
            self.capacity = int(n * 1.25) + 1024
            self.peaks = torch.empty(self.capacity * 24, dtype=torch.uint8, device=self.device)
            self.search_async(prepared, nseries, snr_threshold, stream)
        if max_peaks and n > max_peaks * nseries:
            raise RuntimeError("FFA detection peak count exceeded max_peaks safety guard")
        return n

    def collect(self, prepared: torch.Tensor, nseries: int, snr_threshold: float, max_peaks: int = 0,
                stream=None) -> np.ndarray:
        """Reads the records of the last search_async; on a peak-buffer
        overflow grows the buffer and re-runs, as CudaFfaTileRunner does
        (ffa_cuda_executor.cuh:395-404,491-531)."""
        while True:
            counts = self.counters.cpu()
            if int(counts[1]) & _lib.STATUS_SCHEDULE:
                raise RuntimeError("FFA block schedule exceeded its shared-memory tile")
            n = int(counts[0])
            if n <= self.capacity:
                break
            self.capacity = int(n * 1.25) + 1024
            self.peaks = torch.empty(self.capacity * 24, dtype=torch.uint8, device=self.device)
            self.search_async(prepared, nseries, snr_threshold, stream)
        if max_peaks and n > max_peaks * nseries:
            raise RuntimeError("FFA detection peak count exceeded max_peaks safety guard")
        raw = self.peaks[: n * 24].cpu().numpy()
        return raw.view(_lib.PEAK_RECORD_DTYPE).copy()

    def search(self, prepared: torch.Tensor, nseries: int, snr_threshold: float = 6.0,
               max_peaks: int = 0, stream=None) -> np.ndarray:
        """Transform + detect every task of every series; returns the compact
        peak records (PEAK_RECORD_DTYPE, unordered)."""
        if not math.isfinite(snr_threshold):
            raise ValueError("FFA search S/N threshold must be finite")
        self.search_async(prepared, nseries, snr_threshold, stream)
        return self.collect(prepared, nseries, snr_threshold, max_peaks, stream)

    def expand(self, records: np.ndarray, series_offset: int = 0, dm_low: float = 0.0,
               dm_step: float = 0.0) -> np.ndarray:
        records = np.ascontiguousarray(records, _lib.PEAK_RECORD_DTYPE)
        out = np.zeros(len(records), _lib.PEAK_DTYPE)
        check(_lib.lib().gf_ffa_expand_peaks(self._h, ptr(records), len(records), series_offset, dm_low, dm_step,
                                             ptr(out)))
        return out


class FfaBatchProgram:
    """The FFA plans of many observations (members) as one program
    (gf_ffa_batch_*): one persistent launch per class searches every member's
    series.  members: [(FfaPlan, nseries)].  The prepared buffers are bound
    once, so prepare() and search_async() can be captured in a CUDA graph."""

    def __init__(self, members, device_id: int = 0, prepared=None, scratch=None):
        """prepared (optional): one float32 [nseries][prepared_floats] buffer
        per member (views of a shared arena, say); scratch (optional): a
        uint8 buffer of at least scratch_bytes, or False to attach one later
        with use_scratch (programs that run one after another share one)."""
        self.device = _require_cuda(device_id)
        members = list(members)
        if not members:
            raise ValueError("a batched FFA program needs at least one member")
        self.plans = [m[0] for m in members]
        self.nseries = [int(m[1]) for m in members]
        arr = (_lib.FfaBatchMember * len(members))()
        self._keep = []
        for i, (plan, nseries) in enumerate(members):
            widths = np.ascontiguousarray(plan.width_trials, np.uint64)
            tasks = np.ascontiguousarray(plan.tasks)
            self._keep += [widths, tasks]
            arr[i].tasks, arr[i].ntasks = tasks.ctypes.data, len(tasks)
            arr[i].widths, arr[i].nwidths = widths.ctypes.data, len(widths)
            arr[i].nseries = nseries
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_create(arr, len(members), device_id, C.byref(h)))
        self._h = h
        self.info = _lib.FfaInfo()
        check(_lib.lib().gf_ffa_program_info(h, C.byref(self.info)))
        self.member_info = []
        for i in range(len(members)):
            mi = _lib.FfaMemberInfo()
            check(_lib.lib().gf_ffa_batch_member_info(h, i, C.byref(mi)))
            self.member_info.append(mi)
        if prepared is None:
            prepared = [torch.empty((int(mi.nseries), int(mi.prepared_floats)), dtype=torch.float32,
                                    device=self.device) for mi in self.member_info]
        for t, mi in zip(prepared, self.member_info):
            if t.dtype != torch.float32 or t.numel() < mi.nseries * mi.prepared_floats:
                raise ValueError("prepared buffer too small for its member")
        self.prepared = list(prepared)
        ptrs = (C.c_void_p * len(members))(*[t.data_ptr() for t in self.prepared])
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_bind(h, ptrs))
        self.scratch = None
        if scratch is None:
            scratch = torch.empty(max(16, int(self.info.scratch_bytes)), dtype=torch.uint8, device=self.device)
        if scratch is not False:
            self.use_scratch(scratch)
        self.counters = torch.zeros(2, dtype=torch.int64, device=self.device)
        self.capacity = 1 << 16
        self.peaks = torch.empty(self.capacity * 24, dtype=torch.uint8, device=self.device)

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h and _lib is not None and _lib._lib is not None:
            _lib._lib.gf_ffa_program_destroy(h)

    __del__ = close

    @property
    def kernel_launches(self) -> int:
        return int(self.info.nclasses)

    @property
    def scratch_bytes(self) -> int:
        return int(self.info.scratch_bytes)

    def use_scratch(self, scratch: torch.Tensor) -> None:
        """Search scratch (programs that run one after another may share one)."""
        if scratch.numel() * scratch.element_size() < self.info.scratch_bytes:
            raise ValueError("FFA scratch too small")
        self.scratch = scratch

    def prepare(self, member: int, series: torch.Tensor, stats: torch.Tensor, stream=None) -> None:
        """prepare_ffa_input_cuda of the member's nseries rows of series."""
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_prepare(self._h, member, ptr(series), series.stride(0), ptr(stats),
                                                  _stream(stream)))

    def bind_series(self, series, stats) -> None:
        """The inputs prepare_all reads: per member a float32 [nseries][stride]
        series view and its FP64 [nseries][2] statistics (None: no
        normalisation).  Pointers are fixed here (capturable launches)."""
        n = len(self.prepared)
        if len(series) != n or len(stats) != n:
            raise ValueError("one series view and one statistics table per member")
        for t in series:
            if t.dtype != torch.float32 or t.dim() != 2:
                raise TypeError("series views must be float32 [nseries][stride]")
        sp = (C.c_void_p * n)(*[t.data_ptr() for t in series])
        st = (_lib.u64 * n)(*[t.stride(0) for t in series])
        ss = (C.c_void_p * n)(*[(t.data_ptr() if t is not None else None) for t in stats])
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_bind_series(self._h, sp, st, ss))
        self._bound_series = (list(series), list(stats))

    def prepare_all(self, stream=None) -> None:
        """prepare() of every member, in one launch (after bind_series)."""
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_prepare_all(self._h, _stream(stream)))

    def search_async(self, snr_threshold: float, stream=None) -> None:
        if self.scratch is None:
            raise RuntimeError("batched FFA program has no scratch: call use_scratch")
        with torch.cuda.device(self.device):
            check(_lib.lib().gf_ffa_batch_search(self._h, snr_threshold, ptr(self.scratch), ptr(self.peaks),
                                                 self.capacity, ptr(self.counters), _stream(stream)))

    def collect(self, snr_threshold: float, rerun=None) -> np.ndarray:
        """Records of the last search; on a peak-buffer overflow grows the
        buffer and calls rerun() (default: search_async again)."""
        while True:
            counts = self.counters.cpu()
            if int(counts[1]) & _lib.STATUS_SCHEDULE:
                raise RuntimeError("FFA block schedule exceeded its shared-memory tile")
            n = int(counts[0])
            if n <= self.capacity:
                break
            self.capacity = int(n * 1.25) + 1024
            self.peaks = torch.empty(self.capacity * 24, dtype=torch.uint8, device=self.device)
            (rerun or (lambda: self.search_async(snr_threshold)))()
        raw = self.peaks[: n * 24].cpu().numpy()
        return raw.view(_lib.PEAK_RECORD_DTYPE).copy()

    def expand(self, records: np.ndarray, series_offset, dm_low, dm_step) -> tuple[np.ndarray, np.ndarray]:
        """(peaks, member of each peak); series_offset / dm_low / dm_step per member."""
        records = np.ascontiguousarray(records, _lib.PEAK_RECORD_DTYPE)
        out = np.zeros(len(records), _lib.PEAK_DTYPE)
        member = np.zeros(len(records), np.uint32)
        so = np.ascontiguousarray(series_offset, np.uint64)
        lo = np.ascontiguousarray(dm_low, np.float64)
        st = np.ascontiguousarray(dm_step, np.float64)
        check(_lib.lib().gf_ffa_batch_expand_peaks(self._h, ptr(records), len(records), ptr(so), ptr(lo), ptr(st),
                                                   ptr(out), ptr(member)))
        return out, member


def ffa_transform(x: torch.Tensor, bins: int, stream=None) -> torch.Tensor:
    """Materialised FFA transform of the first rows*bins samples (ffa_transform_cpu,
    src/gaffa/ffa.cpp:389-417) on the device."""
    rows = x.numel() // bins
    out = torch.empty((rows, bins), dtype=torch.float32, device=x.device)
    scratch = torch.empty(2 * rows * bins, dtype=torch.float32, device=x.device)
    src = x.reshape(-1)[: rows * bins].contiguous()
    with torch.cuda.device(x.device):
        check(_lib.lib().gf_ffa_transform(ptr(src), rows, bins, ptr(out), ptr(scratch), _stream(stream)))
    return out


# ---------------------------------------------------------------------------
# host post-processing
# ---------------------------------------------------------------------------

def sort_peaks(peaks: np.ndarray) -> np.ndarray:
    peaks = np.ascontiguousarray(peaks, _lib.PEAK_DTYPE).copy()
    check(_lib.lib().gf_sort_peaks(ptr(peaks), len(peaks)))
    return peaks


def select_candidates(peaks: np.ndarray, observation_seconds: float, frequency_cluster_radius: float = 0.1,
                      dm_cluster_radius: int = 1, cluster_across_widths: bool = True,
                      max_candidates: int = 0) -> np.ndarray:
    """select_candidates_cpu (src/gaffa/candidate.cpp:175-212)."""
    peaks = np.ascontiguousarray(peaks, _lib.PEAK_DTYPE)
    o = _lib.CandidateOptions(frequency_cluster_radius, dm_cluster_radius, int(cluster_across_widths), 0,
                              max_candidates)
    n = _lib.u64()
    check(_lib.lib().gf_select_candidates(ptr(peaks), len(peaks), observation_seconds, C.byref(o), None, 0,
                                          C.byref(n)))
    out = np.zeros(n.value, _lib.CAND_DTYPE)
    check(_lib.lib().gf_select_candidates(ptr(peaks), len(peaks), observation_seconds, C.byref(o), ptr(out),
                                          len(out), C.byref(n)))
    return out


def select_candidates_device(program: "FfaProgram", records: torch.Tensor, segments, dm_low: float, dm_step: float,
                             observation_seconds: float, frequency_cluster_radius: float = 0.1,
                             dm_cluster_radius: int = 1, cluster_across_widths: bool = True,
                             max_candidates: int = 0, stream=None) -> np.ndarray:
    """select_candidates_cpu (src/gaffa/candidate.cpp:175-212) over compact
    device peak records (uint8 tensor of 24-byte records) without expanding
    them on the host: segments are (record_begin, record_count, dm_offset)
    runs of records of one FfaProgram search each.  Equals select_candidates
    of the expanded, sorted peaks."""
    segs = list(segments)
    arr = (_lib.PeakSegment * max(1, len(segs)))()
    total = 0
    for i, (b, n, off) in enumerate(segs):
        arr[i] = _lib.PeakSegment(int(b), int(n), int(off))
        total += int(n)
    o = _lib.CandidateOptions(frequency_cluster_radius, dm_cluster_radius, int(cluster_across_widths), 0,
                              max_candidates)
    if total == 0:
        return np.zeros(0, _lib.CAND_DTYPE)
    ws_bytes = _lib.u64()
    with torch.cuda.device(program.device):
        check(_lib.lib().gf_select_candidates_device_workspace(total, C.byref(ws_bytes)))
        ws = torch.empty(int(ws_bytes.value), dtype=torch.uint8, device=program.device)
        n = _lib.u64()
        # usually far fewer candidates than peaks: a bounded first guess, and a
        # second call only when the candidates exceed it
        out = np.zeros(min(total, 1 << 16), _lib.CAND_DTYPE)
        for _ in range(2):
            check(_lib.lib().gf_select_candidates_device(program._h, ptr(records), arr, len(segs), dm_low, dm_step,
                                                         observation_seconds, C.byref(o), ptr(ws), ws.numel(),
                                                         ptr(out), len(out), C.byref(n), _stream(stream)))
            if n.value <= len(out):
                break
            out = np.zeros(n.value, _lib.CAND_DTYPE)
    return out[: n.value]


def dedisperse_spectrum(filterbank: torch.Tensor, frequency_mhz, dm: float, tsamp: float,
                        ref_frequency_mhz: float | None = None, chan_begin: int = 0, chan_end: int | None = None,
                        stream=None) -> torch.Tensor:
    """dedisperse_spectrum_cpu / _cuda (src/gaffa/dedispersion.cpp:249-289) on a
    device-resident time-major [nsamples][nchans] filterbank (uint8, int16
    holding uint16, or float32): [nout][chan_end - chan_begin], each channel
    shifted by its delay at dm."""
    if filterbank.dim() != 2 or not filterbank.is_cuda:
        raise ValueError("filterbank must be a 2-D CUDA tensor [nsamples][nchans]")
    elem = {torch.uint8: 1, torch.int16: 2, torch.uint16: 2, torch.float32: 4}.get(filterbank.dtype)
    if elem is None:
        raise TypeError("filterbank dtype must be uint8, uint16 or float32")
    fb = filterbank.contiguous()
    freq = np.ascontiguousarray(frequency_mhz, dtype=np.float64)
    nsamples, nchans = fb.shape
    ref = float(freq.max()) if ref_frequency_mhz is None else ref_frequency_mhz
    ce = nchans if chan_end is None else chan_end
    nout = _lib.u64()
    fptr = freq.ctypes.data_as(C.POINTER(C.c_double))
    check(_lib.lib().gf_dedisperse_spectrum(None, elem, nsamples, nchans, fptr, dm, ref, tsamp, chan_begin, ce,
                                            None, C.byref(nout), None))
    out = torch.empty((nout.value, ce - chan_begin), dtype=fb.dtype, device=fb.device)
    s = stream if stream is not None else torch.cuda.current_stream(fb.device)
    check(_lib.lib().gf_dedisperse_spectrum(ptr(fb), elem, nsamples, nchans, fptr, dm, ref, tsamp, chan_begin, ce,
                                            ptr(out), C.byref(nout), C.c_void_p(s.cuda_stream)))
    return out


# ---------------------------------------------------------------------------
# filterbank ingest
# ---------------------------------------------------------------------------

_FB_DTYPE = {8: np.uint8, 16: np.uint16, 32: np.float32}


def read_filterbank_header(path, preserve_file_order: bool = False) -> tuple[dict, np.ndarray]:
    """read_filterbank's header (src/gaffa/io/filterbank.cpp:116-224, 335-348):
    the normalised fields and the delivered channels' frequencies."""
    h = _lib.FilterbankHeader()
    order = _lib.CHANNEL_ORDER_FILE if preserve_file_order else _lib.CHANNEL_ORDER_ASCENDING
    p = str(path).encode()
    check(_lib.lib().gf_filterbank_read_header(p, order, C.byref(h), None, 0))
    freq = np.zeros(h.nchans, np.float64)
    check(_lib.lib().gf_filterbank_read_header(p, order, C.byref(h), ptr(freq), len(freq)))
    fields = {k: getattr(h, k) for k, _ in h._fields_}
    fields["rawdatafile"] = h.rawdatafile.decode()
    fields["source_name"] = h.source_name.decode()
    return fields, freq


def _fb_shape(h: dict, nrows: int) -> tuple[tuple, object]:
    nbits = h["nbits"]
    if nbits in _FB_DTYPE:
        return (nrows, h["nifs"], h["nchans"]), _FB_DTYPE[nbits]
    return (nrows, h["nifs"], h["nchans"] * nbits // 8), np.uint8  # packed rows


def read_filterbank(path, preserve_file_order: bool = False, row_begin: int = 0, nrows: int | None = None):
    """read_filterbank into host memory: (header, frequencies, samples
    [nrows][nifs][nchans] (packed bytes for nbits < 8))."""
    h, freq = read_filterbank_header(path, preserve_file_order)
    n = h["nsamples"] - row_begin if nrows is None else nrows
    shape, dt = _fb_shape(h, n)
    out = np.zeros(shape, dt)
    order = _lib.CHANNEL_ORDER_FILE if preserve_file_order else _lib.CHANNEL_ORDER_ASCENDING
    check(_lib.lib().gf_filterbank_read_host(str(path).encode(), order, row_begin, n, ptr(out) if out.size else None))
    return h, freq, out


def load_filterbank(path, preserve_file_order: bool = False, row_begin: int = 0, nrows: int | None = None,
                    device_id: int = 0, bounce_bytes: int = 64 << 20, stream=None):
    """The same samples loaded straight into device memory: file reads through
    a pinned bounce buffer overlap the host-to-device copies, and the channel
    reversal runs on the GPU.  Returns (header, frequencies, device tensor)."""
    h, freq = read_filterbank_header(path, preserve_file_order)
    n = h["nsamples"] - row_begin if nrows is None else nrows
    shape, dt = _fb_shape(h, n)
    tdt = {np.uint8: torch.uint8, np.uint16: torch.int16, np.float32: torch.float32}[dt]
    dev = torch.device("cuda", device_id)
    out = torch.empty(shape, dtype=tdt, device=dev)
    bounce = torch.empty(max(bounce_bytes, 2 * int(np.prod(shape[1:])) * np.dtype(dt).itemsize), dtype=torch.uint8,
                         pin_memory=True)
    order = _lib.CHANNEL_ORDER_FILE if preserve_file_order else _lib.CHANNEL_ORDER_ASCENDING
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        check(_lib.lib().gf_filterbank_load(str(path).encode(), order, row_begin, n, ptr(out) if out.numel() else None,
                                            ptr(bounce), bounce.numel(), C.c_void_p(s.cuda_stream)))
    s.synchronize()  # the bounce buffer is released on return
    return h, freq, out


def fold_spectrum(spectrum: torch.Tensor, period: float, tsamp: float, nbin: int, subint_samples: int,
                  start_sample: int = 0, output_channels: int = 0, stream=None):
    """fold_spectrum_cpu (src/gaffa/folding.cpp:300-420) on a device spectrum
    [nsamples][nchans]: (cube [nsubint][nout][nbin] float, exposure
    [nsubint][nbin] double), both on the device."""
    if spectrum.dim() != 2 or not spectrum.is_cuda:
        raise ValueError("spectrum must be a 2-D CUDA tensor [nsamples][nchans]")
    elem = {torch.uint8: 1, torch.int16: 2, torch.uint16: 2, torch.float32: 4}.get(spectrum.dtype)
    if elem is None:
        raise TypeError("spectrum dtype must be uint8, uint16 or float32")
    sp = spectrum.contiguous()
    ns, nc = sp.shape
    nout = output_channels or nc
    nsub = -(-ns // subint_samples) if subint_samples > 0 else 0
    cube = torch.empty((max(nsub, 1), nout, nbin), dtype=torch.float32, device=sp.device)
    expo = torch.empty((max(nsub, 1), nbin), dtype=torch.float64, device=sp.device)
    status = torch.empty(1, dtype=torch.int32, device=sp.device)
    s = stream if stream is not None else torch.cuda.current_stream(sp.device)
    check(_lib.lib().gf_fold_spectrum(ptr(sp), elem, ns, nc, period, tsamp, nbin, subint_samples, start_sample,
                                      output_channels, ptr(cube), ptr(expo), ptr(status), C.c_void_p(s.cuda_stream)))
    if int(status.item()) & _lib.STATUS_NONFINITE:
        raise ValueError("fold spectrum must contain only finite samples")
    return cube, expo


def fold_dedispersed_spectrum(filterbank: torch.Tensor, frequency_mhz, dm: float, period: float, tsamp: float,
                              nbin: int, tsubint: float = 10.0, output_channels: int = 0):
    """fold_dedispersed_spectrum (src/gaffa/folding.cpp:408-438): aligned
    spectrum at dm, folded into subints of round(tsubint / tsamp) samples, and
    the projections.  Returns a dict of device tensors."""
    if not (math.isfinite(tsubint) and tsubint > 0.0):
        raise ValueError("fold tsubint must be finite and positive")
    sub = max(1, int(round(tsubint / tsamp)))
    spec = dedisperse_spectrum(filterbank, frequency_mhz, dm, tsamp)
    cube, expo = fold_spectrum(spec, period, tsamp, nbin, sub, 0, output_channels)
    nsub, nch, _ = cube.shape
    prof = torch.empty(nbin, dtype=torch.float32, device=cube.device)
    fp = torch.empty((nch, nbin), dtype=torch.float32, device=cube.device)
    tp = torch.empty((nsub, nbin), dtype=torch.float32, device=cube.device)
    s = torch.cuda.current_stream(cube.device)
    check(_lib.lib().gf_project_folded_cube(ptr(cube), ptr(expo), nsub, nch, nbin, ptr(prof), ptr(fp), ptr(tp),
                                            C.c_void_p(s.cuda_stream)))
    return {"cube": cube, "exposure": expo, "profile": prof, "freq_phase": fp, "time_phase": tp,
            "tsubint": sub * tsamp}


def harmonic_options(max_harmonic: int = 16, denominator_max: int = 5, frequency_tolerance_bins: float = 1.5,
                     phase_distance_max: float = 1.0, dm_distance_max: float = 3.0,
                     use_snr_consistency: bool = False, snr_distance_max: float = 3.0):
    """HarmonicOptions (include/gaffa/harmonic.h:22-36) with its defaults."""
    return _lib.HarmonicOptions(max_harmonic, denominator_max, frequency_tolerance_bins, phase_distance_max,
                                dm_distance_max, int(use_snr_consistency), 0, snr_distance_max)


# candidate counts from which harmonic flagging runs its pairwise tests on the GPU
DEVICE_HARMONIC_MIN = 4096


def flag_harmonics(candidates: np.ndarray, observation_seconds: float, frequency_low_mhz: float,
                   frequency_high_mhz: float, options=None, device_id: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """flag_harmonics_cpu (src/gaffa/harmonic.cpp:245-292): the candidates in
    harmonic ranking order and their relations (HARMONIC_DTYPE).  The n^2/2
    pairwise tests run on the GPU (gf_flag_harmonics_device, same decisions)
    when device_id is given, or from DEVICE_HARMONIC_MIN candidates on."""
    candidates = np.ascontiguousarray(candidates, _lib.CAND_DTYPE)
    ctx = _lib.HarmonicContext(observation_seconds, frequency_low_mhz, frequency_high_mhz)
    opts = options if options is not None else harmonic_options()
    out = np.zeros(len(candidates), _lib.CAND_DTYPE)
    rel = np.zeros(len(candidates), _lib.HARMONIC_DTYPE)
    if device_id is None and len(candidates) >= DEVICE_HARMONIC_MIN and torch.cuda.is_available():
        device_id = torch.cuda.current_device()
    if device_id is None:
        check(_lib.lib().gf_flag_harmonics(ptr(candidates), len(candidates), C.byref(ctx), C.byref(opts),
                                           ptr(out) if len(out) else None, ptr(rel) if len(rel) else None))
    else:
        with torch.cuda.device(device_id):
            check(_lib.lib().gf_flag_harmonics_device(ptr(candidates), len(candidates), C.byref(ctx), C.byref(opts),
                                                      ptr(out) if len(out) else None, ptr(rel) if len(rel) else None,
                                                      device_id, _stream()))
    return out, rel


def remove_harmonics(sorted_candidates: np.ndarray, relations: np.ndarray, max_candidates: int = 0) -> np.ndarray:
    """remove_harmonics_cpu (src/gaffa/harmonic.cpp:294-309)."""
    sorted_candidates = np.ascontiguousarray(sorted_candidates, _lib.CAND_DTYPE)
    relations = np.ascontiguousarray(relations, _lib.HARMONIC_DTYPE)
    if len(sorted_candidates) != len(relations):
        raise ValueError("candidates and relations must have the same length")
    out = np.zeros(len(sorted_candidates), _lib.CAND_DTYPE)
    n = _lib.u64()
    check(_lib.lib().gf_remove_harmonics(ptr(sorted_candidates) if len(out) else None,
                                         ptr(relations) if len(out) else None, len(out), max_candidates,
                                         ptr(out) if len(out) else None, C.byref(n)))
    return out[: n.value]


# ---------------------------------------------------------------------------
# folding
# ---------------------------------------------------------------------------

def fold_time_series(series: torch.Tensor, period: float, tsamp: float, nbin: int, start_sample: int = 0,
                     stream=None):
    """fold_time_series_cpu (src/gaffa/folding.cpp:452-502) on a device series
    (uint32 stored as int32, or float32).  Returns host (profile, exposure)."""
    if series.dim() != 1:
        series = series.reshape(-1)
    is_u32 = series.dtype in (torch.int32, torch.uint32)
    n = series.numel()
    ws_bytes = int(_lib.lib().gf_fold_workspace_bytes(n, nbin))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=series.device)
    prof = torch.empty(nbin, dtype=torch.float32, device=series.device)
    expo = torch.empty(nbin, dtype=torch.float64, device=series.device)
    with torch.cuda.device(series.device):
        check(_lib.lib().gf_fold_time_series(ptr(series), int(is_u32), n, period, tsamp, nbin, start_sample,
                                             ptr(prof), ptr(expo), ptr(ws), _stream(stream)))
    status = int(ws[ws_bytes - 16: ws_bytes - 12].view(torch.int32).item())
    if status & _lib.STATUS_NONFINITE:
        raise ValueError("fold input must contain only finite samples")
    return prof.cpu().numpy(), expo.cpu().numpy()


# ---------------------------------------------------------------------------
# synthetic observations
# ---------------------------------------------------------------------------

def synth_generate(obs, t_begin: int = 0, t_end: int | None = None, out: torch.Tensor | None = None,
                   device_id: int = 0, stream=None) -> torch.Tensor:
    """The synth.py observation generated on the device (same noise bits)."""
    from . import synth
    device = _require_cuda(device_id)
    t_end = obs.nsamples if t_end is None else t_end
    row = obs.nchans if obs.nbits == 8 else obs.nchans // 4
    if out is None:
        out = torch.empty((t_end - t_begin, row), dtype=torch.uint8, device=device)
    ps = (_lib.SynthPulsar * max(1, len(obs.pulsars)))()
    for i, p in enumerate(obs.pulsars):
        ps[i] = _lib.SynthPulsar(p.period, p.dm, p.duty_cycle, p.amplitude, p.phase)
    d = _lib.SynthDesc()
    d.nchans, d.nsamples, d.tsamp = obs.nchans, obs.nsamples, obs.tsamp
    d.f_low, d.f_high, d.nbits = obs.f_low, obs.f_high, obs.nbits
    d.npulsars, d.seed = len(obs.pulsars), obs.seed
    d.pulsars = C.cast(ps, C.POINTER(_lib.SynthPulsar))
    r = obs.rfi
    d.narrowband_fraction, d.narrowband_hz, d.narrowband_amplitude = (r.narrowband_fraction, r.narrowband_hz,
                                                                      r.narrowband_amplitude)
    d.impulse_hz, d.impulse_amplitude = r.impulse_hz, r.impulse_amplitude
    mask = None
    if r.narrowband_fraction > 0.0:
        mask = np.ascontiguousarray(synth._narrowband_mask(obs).astype(np.uint8))
        d.narrowband_mask = mask.ctypes.data_as(C.POINTER(C.c_uint8))
    with torch.cuda.device(device):
        check(_lib.lib().gf_synth_generate(C.byref(d), t_begin, t_end, ptr(out), _stream(stream)))
    return out
