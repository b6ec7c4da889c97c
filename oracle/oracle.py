"""ctypes access to the CPU checkers (TEST INFRASTRUCTURE ONLY).

``Oracle("port")`` loads ``oracle/libgaffa_oracle.so`` -- the C restatement of
the reference CPU path in ``gaffa_oracle.c``.  ``Oracle("reference")`` loads
``oracle/_ref/libgaffa_ref.so`` -- the reference's own CPU sources compiled in
place with ``ref_shim.cpp``.  Both expose identical functions, so tests can
compare them bit for bit.  Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "libgaffa_oracle.so"
REF_LIB = HERE / "_ref" / "libgaffa_ref.so"

TASK_DTYPE = np.dtype([
    ("downsample_factor", "<f8"), ("effective_tsamp", "<f8"),
    ("input_nsamples", "<u8"), ("prepared_nsamples", "<u8"), ("bins", "<u8"),
    ("rows", "<u8"), ("rows_eval", "<u8"), ("period_begin", "<f8"),
    ("period_end", "<f8"),
])
PEAK_DTYPE = np.dtype([
    ("dm", "<f8"), ("dm_index", "<u8"), ("period", "<f8"), ("frequency", "<f8"),
    ("width", "<u8"), ("duty_cycle", "<f8"), ("width_index", "<u8"),
    ("period_index", "<u8"), ("phase", "<u8"), ("shift", "<u8"), ("bins", "<u8"),
    ("snr", "<f4"), ("reserved", "<u4"),
])
CAND_DTYPE = np.dtype([
    ("dm", "<f8"), ("dm_index", "<u8"), ("period", "<f8"), ("frequency", "<f8"),
    ("width", "<u8"), ("duty_cycle", "<f8"), ("snr", "<f4"), ("reserved", "<u4"),
    ("peak_count", "<u8"), ("dm_index_min", "<u8"), ("dm_index_max", "<u8"),
    ("frequency_min", "<f8"), ("frequency_max", "<f8"), ("best_peak", PEAK_DTYPE),
])


class PlanOptions(C.Structure):
    _fields_ = [("period_min", C.c_double), ("period_max", C.c_double),
                ("bins_min", C.c_uint64), ("bins_max", C.c_uint64),
                ("min_periods", C.c_uint64), ("duty_cycle_max", C.c_double),
                ("width_trial_spacing", C.c_double), ("max_tasks", C.c_uint64)]


class PreprocessOptions(C.Structure):
    _fields_ = [("window_seconds", C.c_double), ("min_points", C.c_uint64),
                ("normalise", C.c_int32), ("reject_constant", C.c_int32)]


HARMONIC_DTYPE = np.dtype([
    ("is_harmonic", "<i4"), ("reserved", "<i4"), ("parent_index", "<u8"), ("numerator", "<i4"),
    ("denominator", "<i4"), ("frequency_error_bins", "<f8"), ("phase_distance", "<f8"),
    ("dm_distance", "<f8"), ("expected_snr", "<f8"), ("snr_distance", "<f8")])


class HarmonicContext(C.Structure):
    _fields_ = [("observation_seconds", C.c_double), ("frequency_low_mhz", C.c_double),
                ("frequency_high_mhz", C.c_double)]


class HarmonicOptions(C.Structure):
    _fields_ = [("max_harmonic", C.c_uint64), ("denominator_max", C.c_uint64),
                ("frequency_tolerance_bins", C.c_double), ("phase_distance_max", C.c_double),
                ("dm_distance_max", C.c_double), ("use_snr_consistency", C.c_int32),
                ("reserved", C.c_int32), ("snr_distance_max", C.c_double)]


class CandidateOptions(C.Structure):
    _fields_ = [("frequency_cluster_radius", C.c_double),
                ("dm_cluster_radius", C.c_uint64),
                ("cluster_across_widths", C.c_int32), ("reserved", C.c_int32),
                ("max_candidates", C.c_uint64)]


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


def build(ref_dir: str | None = None) -> None:
    """Compile the port and, when ``ref_dir`` (or the GAFFA_REFERENCE_DIR
    environment variable) names a gaffa checkout, the reference."""
    env = dict(os.environ)
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True, env=env)
    ref = ref_dir or os.environ.get("GAFFA_REFERENCE_DIR")
    if ref and Path(ref, "src", "gaffa").is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_DIR={ref}"],
                       check=True, env=env)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class Oracle:
    """One of the two CPU implementations, with numpy-facing helpers."""

    def __init__(self, kind: str = "port"):
        self.kind = kind
        path = PORT_LIB if kind == "port" else REF_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (make -C oracle)")
        self.lib = C.CDLL(str(path))
        self.p = "gfo_" if kind == "port" else "gfr_"
        self._fn("last_error").restype = C.c_char_p

    @staticmethod
    def available(kind: str) -> bool:
        return (PORT_LIB if kind == "port" else REF_LIB).exists()

    def _fn(self, name):
        return getattr(self.lib, self.p + name)

    def _check(self, rc):
        if rc != 0:
            raise OracleError(rc, self._fn("last_error")().decode())

    def _take(self, ptr, n, dtype):
        if n == 0:
            self._fn("free")(ptr)
            return np.zeros(0, dtype)
        buf = C.cast(ptr, C.POINTER(C.c_uint8 * (n * dtype.itemsize))).contents
        out = np.frombuffer(bytes(buf), dtype=dtype).copy()
        self._fn("free")(ptr)
        return out

    # ---- dedispersion -------------------------------------------------------
    def output_nsamples(self, freq, nsamples, dm_low, dm_step, ndm, fref, tsamp,
                        chan_begin=0, chan_end=None):
        freq = np.ascontiguousarray(freq, np.float64)
        chan_end = len(freq) if chan_end is None else chan_end
        n = C.c_uint64()
        f = getattr(PORT_LIB_HANDLE(), "gfo_multi_dm_output_nsamples")
        rc = f(_ptr(freq, C.c_double), C.c_uint64(len(freq)), C.c_uint64(nsamples),
               C.c_double(dm_low), C.c_double(dm_step), C.c_uint64(ndm),
               C.c_double(fref), C.c_double(tsamp), C.c_uint64(chan_begin),
               C.c_uint64(chan_end), C.byref(n))
        if rc:
            raise OracleError(rc, PORT_LIB_HANDLE().gfo_last_error().decode())
        return n.value

    def dedisperse_multi_dm(self, data, freq, dm_low, dm_step, ndm, fref, tsamp,
                            chan_begin=0, chan_end=None):
        data = np.ascontiguousarray(data, np.uint8)
        ns, nc = data.shape
        chan_end = nc if chan_end is None else chan_end
        nout = self.output_nsamples(freq, ns, dm_low, dm_step, ndm, fref, tsamp,
                                    chan_begin, chan_end)
        out = np.zeros((ndm, nout), np.uint32)
        freq = np.ascontiguousarray(freq, np.float64)
        self._check(self._fn("dedisperse_multi_dm_u8")(
            _ptr(data, C.c_uint8), C.c_uint64(ns), C.c_uint64(nc),
            _ptr(freq, C.c_double), C.c_double(dm_low), C.c_double(dm_step),
            C.c_uint64(ndm), C.c_double(fref), C.c_double(tsamp),
            C.c_uint64(chan_begin), C.c_uint64(chan_end), _ptr(out, C.c_uint32)))
        return out

    def dedisperse_subband(self, data, freq, dm_low, dm_step, ndm, fref, tsamp,
                           subband_channels=32, ndm_per_nominal=32, chan_begin=0,
                           chan_end=None):
        data = np.ascontiguousarray(data, np.uint8)
        ns, nc = data.shape
        chan_end = nc if chan_end is None else chan_end
        nout = self.output_nsamples(freq, ns, dm_low, dm_step, ndm, fref, tsamp,
                                    chan_begin, chan_end)
        out = np.zeros((ndm, nout), np.uint32)
        freq = np.ascontiguousarray(freq, np.float64)
        self._check(self._fn("dedisperse_subband_u8")(
            _ptr(data, C.c_uint8), C.c_uint64(ns), C.c_uint64(nc),
            _ptr(freq, C.c_double), C.c_double(dm_low), C.c_double(dm_step),
            C.c_uint64(ndm), C.c_double(fref), C.c_double(tsamp),
            C.c_uint64(chan_begin), C.c_uint64(chan_end),
            C.c_uint64(subband_channels), C.c_uint64(ndm_per_nominal),
            _ptr(out, C.c_uint32)))
        return out

    # ---- time series / preprocessing ----------------------------------------
    def downsample(self, x, factor):
        x = np.ascontiguousarray(x, np.float32)
        m = int(np.floor(len(x) / factor))
        out = np.zeros(m, np.float32)
        self._check(self._fn("downsample_weighted_sum")(
            _ptr(x, C.c_float), C.c_uint64(len(x)), C.c_double(factor),
            _ptr(out, C.c_float)))
        return out

    def downsampled_variance(self, n, factor):
        v = C.c_double()
        self._check(self._fn("downsampled_variance")(C.c_uint64(n), C.c_double(factor),
                                                     C.byref(v)))
        return v.value

    def preprocess(self, x, tsamp, window_seconds=1.0, min_points=101,
                   normalise=True, reject_constant=True):
        x = np.array(x, np.float32, copy=True)
        o = PreprocessOptions(window_seconds, min_points, int(normalise),
                              int(reject_constant))
        self._check(self._fn("preprocess_riptide")(
            _ptr(x, C.c_float), C.c_uint64(len(x)), C.c_double(tsamp), C.byref(o)))
        return x

    # ---- FFA ------------------------------------------------------------------
    def make_plan(self, nsamples, tsamp, period_min, period_max, bins_min=180,
                  bins_max=256, min_periods=1, duty_cycle_max=0.2,
                  width_trial_spacing=1.5, max_tasks=1_000_000):
        o = PlanOptions(period_min, period_max, bins_min, bins_max, min_periods,
                        duty_cycle_max, width_trial_spacing, max_tasks)
        tp, nt = C.c_void_p(), C.c_uint64()
        wp, nw = C.c_void_p(), C.c_uint64()
        self._check(self._fn("make_riptide_ffa_plan")(
            C.c_uint64(nsamples), C.c_double(tsamp), C.byref(o), C.byref(tp),
            C.byref(nt), C.byref(wp), C.byref(nw)))
        tasks = self._take(tp, nt.value, TASK_DTYPE)
        widths = self._take(wp, nw.value, np.dtype("<u8"))
        return tasks, widths

    def ffa_transform(self, x, bins):
        x = np.ascontiguousarray(x, np.float32)
        rows = len(x) // bins
        x = np.ascontiguousarray(x[: rows * bins])
        out = np.zeros((rows, bins), np.float32)
        self._check(self._fn("ffa_transform")(_ptr(x, C.c_float), C.c_uint64(rows),
                                              C.c_uint64(bins), _ptr(out, C.c_float)))
        return out

    def ffa_search(self, x, tasks, widths, snr_threshold=6.0, max_peaks=0):
        x = np.ascontiguousarray(x, np.float32)
        tasks = np.ascontiguousarray(tasks, TASK_DTYPE)
        widths = np.ascontiguousarray(widths, np.uint64)
        pp, n = C.c_void_p(), C.c_uint64()
        self._check(self._fn("ffa_search")(
            x.ctypes.data_as(C.POINTER(C.c_float)), C.c_uint64(len(x)),
            tasks.ctypes.data_as(C.c_void_p), C.c_uint64(len(tasks)),
            widths.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_uint64(len(widths)),
            C.c_float(snr_threshold), C.c_uint64(max_peaks), C.byref(pp), C.byref(n)))
        return self._take(pp, n.value, PEAK_DTYPE)

    def find_dm_peaks(self, data, dms, tsamp, plan: dict, preprocess: dict | None,
                      snr_threshold=6.0, max_peaks=0, widths=None):
        data = np.ascontiguousarray(data, np.uint32)
        ndm, ns = data.shape
        dms = np.ascontiguousarray(dms, np.float64)
        po = PlanOptions(plan["period_min"], plan["period_max"],
                         plan.get("bins_min", 180), plan.get("bins_max", 256),
                         plan.get("min_periods", 1), plan.get("duty_cycle_max", 0.2),
                         plan.get("width_trial_spacing", 1.5),
                         plan.get("max_tasks", 1_000_000))
        pre = None
        if preprocess is not None:
            pre = PreprocessOptions(preprocess.get("window_seconds", 1.0),
                                    preprocess.get("min_points", 101),
                                    int(preprocess.get("normalise", True)),
                                    int(preprocess.get("reject_constant", True)))
        w = np.ascontiguousarray(widths if widths is not None else [], np.uint64)
        pp, n = C.c_void_p(), C.c_uint64()
        self._check(self._fn("find_dm_peaks_u32")(
            _ptr(data, C.c_uint32), C.c_uint64(ndm), C.c_uint64(ns),
            _ptr(dms, C.c_double), C.c_double(tsamp), C.byref(po),
            C.byref(pre) if pre is not None else None, C.c_float(snr_threshold),
            C.c_uint64(max_peaks), _ptr(w, C.c_uint64) if len(w) else None,
            C.c_uint64(len(w)), C.byref(pp), C.byref(n)))
        return self._take(pp, n.value, PEAK_DTYPE)

    def select_candidates(self, peaks, observation_seconds,
                          frequency_cluster_radius=0.1, dm_cluster_radius=1,
                          cluster_across_widths=True, max_candidates=0):
        peaks = np.ascontiguousarray(peaks, PEAK_DTYPE)
        o = CandidateOptions(frequency_cluster_radius, dm_cluster_radius,
                             int(cluster_across_widths), 0, max_candidates)
        cp, n = C.c_void_p(), C.c_uint64()
        self._check(self._fn("select_candidates")(
            peaks.ctypes.data_as(C.c_void_p), C.c_uint64(len(peaks)),
            C.c_double(observation_seconds), C.byref(o), C.byref(cp), C.byref(n)))
        return self._take(cp, n.value, CAND_DTYPE)

    def dedisperse_spectrum(self, data, freq, dm, ref, tsamp, chan_begin=0, chan_end=None):
        data = np.ascontiguousarray(data, np.uint8)
        freq = np.ascontiguousarray(freq, np.float64)
        ns, nc = data.shape
        ce = nc if chan_end is None else chan_end
        f = self._fn("dedisperse_spectrum_u8")
        nout = C.c_uint64()
        args = [data.ctypes.data_as(C.c_void_p), C.c_uint64(ns), C.c_uint64(nc),
                freq.ctypes.data_as(C.c_void_p), C.c_double(dm), C.c_double(ref), C.c_double(tsamp),
                C.c_uint64(chan_begin), C.c_uint64(ce)]
        self._check(f(*args, None, C.byref(nout)))
        out = np.zeros((nout.value, ce - chan_begin), np.uint8)
        self._check(f(*args, out.ctypes.data_as(C.c_void_p), C.byref(nout)))
        return out

    def read_filterbank(self, path, preserve_file_order=False):
        """read_filterbank (reference only): (header fields, frequencies, sample bytes)."""
        class Hdr(C.Structure):
            _fields_ = [("header_size", C.c_int64), ("nsamples", C.c_int64)] + \
                [(n, C.c_int32) for n in ("telescope_id", "machine_id", "data_type", "barycentric",
                                          "pulsarcentric", "ibeam", "nbeams", "npuls", "nbins", "nbits",
                                          "nifs", "nchans")] + \
                [(n, C.c_double) for n in ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp",
                                           "fch1", "foff", "refdm", "period")] + \
                [("uses_frequency_table", C.c_int32), ("reversed", C.c_int32),
                 ("rawdatafile", C.c_char * 256), ("source_name", C.c_char * 256)]
        h = Hdr()
        freq = np.zeros(1 << 16, np.float64)
        sp, n = C.c_void_p(), C.c_uint64()
        self._check(self._fn("read_filterbank")(str(path).encode(), int(preserve_file_order), C.byref(h),
                                                freq.ctypes.data_as(C.c_void_p), C.c_uint64(len(freq)),
                                                C.byref(sp), C.byref(n)))
        data = self._take(sp, n.value, np.dtype(np.uint8))
        fields = {k: getattr(h, k) for k, _ in h._fields_ if k not in ("reversed",)}
        fields["rawdatafile"] = h.rawdatafile.decode()
        fields["source_name"] = h.source_name.decode()
        return fields, freq[: h.nchans].copy(), data

    def fold_dedispersed_spectrum(self, spectrum, period, tsamp, nbin, tsubint=10.0, output_channels=0):
        """fold_dedispersed_spectrum_view_cpu of a uint8 [ns][nc] spectrum (reference only)."""
        x = np.ascontiguousarray(spectrum, np.uint8)
        ns, nc = x.shape
        f = self._fn("fold_dedispersed_spectrum_u8")
        nsub = C.c_uint64()
        args = [x.ctypes.data_as(C.c_void_p), C.c_uint64(ns), C.c_uint64(nc), C.c_double(period),
                C.c_double(tsamp), C.c_uint64(nbin), C.c_double(tsubint), C.c_uint64(output_channels),
                C.byref(nsub)]
        self._check(f(*args, None, None, None, None, None))
        nout = output_channels or nc
        out = dict(cube=np.zeros((nsub.value, nout, nbin), np.float32),
                   exposure=np.zeros((nsub.value, nbin), np.float64), profile=np.zeros(nbin, np.float32),
                   freq_phase=np.zeros((nout, nbin), np.float32), time_phase=np.zeros((nsub.value, nbin), np.float32))
        self._check(f(*args, *[out[k].ctypes.data_as(C.c_void_p) for k in
                               ("cube", "exposure", "profile", "freq_phase", "time_phase")]))
        return out

    def flag_harmonics(self, candidates, observation_seconds, frequency_low_mhz, frequency_high_mhz,
                       max_harmonic=16, denominator_max=5, frequency_tolerance_bins=1.5,
                       phase_distance_max=1.0, dm_distance_max=3.0, use_snr_consistency=False,
                       snr_distance_max=3.0):
        candidates = np.ascontiguousarray(candidates, CAND_DTYPE)
        ctx = HarmonicContext(observation_seconds, frequency_low_mhz, frequency_high_mhz)
        o = HarmonicOptions(max_harmonic, denominator_max, frequency_tolerance_bins, phase_distance_max,
                            dm_distance_max, int(use_snr_consistency), 0, snr_distance_max)
        out = np.zeros(len(candidates), CAND_DTYPE)
        rel = np.zeros(len(candidates), HARMONIC_DTYPE)
        self._check(self._fn("flag_harmonics")(
            candidates.ctypes.data_as(C.c_void_p), C.c_uint64(len(candidates)), C.byref(ctx), C.byref(o),
            out.ctypes.data_as(C.c_void_p), rel.ctypes.data_as(C.c_void_p)))
        return out, rel

    def remove_harmonics(self, sorted_candidates, relations, max_candidates=0):
        sorted_candidates = np.ascontiguousarray(sorted_candidates, CAND_DTYPE)
        relations = np.ascontiguousarray(relations, HARMONIC_DTYPE)
        out = np.zeros(len(sorted_candidates), CAND_DTYPE)
        n = C.c_uint64()
        self._check(self._fn("remove_harmonics")(
            sorted_candidates.ctypes.data_as(C.c_void_p), relations.ctypes.data_as(C.c_void_p),
            C.c_uint64(len(out)), C.c_uint64(max_candidates), out.ctypes.data_as(C.c_void_p), C.byref(n)))
        return out[: n.value]

    def fold(self, x, period, tsamp, nbin, start_sample=0):
        x = np.ascontiguousarray(x)
        prof = np.zeros(nbin, np.float32)
        expo = np.zeros(nbin, np.float64)
        if x.dtype == np.uint32:
            f, pt = self._fn("fold_time_series_u32"), C.c_uint32
        else:
            x = np.ascontiguousarray(x, np.float32)
            f, pt = self._fn("fold_time_series_f32"), C.c_float
        self._check(f(_ptr(x, pt), C.c_uint64(len(x)), C.c_double(period),
                      C.c_double(tsamp), C.c_uint64(nbin), C.c_uint64(start_sample),
                      _ptr(prof, C.c_float), _ptr(expo, C.c_double)))
        return prof, expo


_PORT_HANDLE = None


def PORT_LIB_HANDLE():
    """The port library (shared helpers such as the output length)."""
    global _PORT_HANDLE
    if _PORT_HANDLE is None:
        _PORT_HANDLE = C.CDLL(str(PORT_LIB))
        _PORT_HANDLE.gfo_last_error.restype = C.c_char_p
    return _PORT_HANDLE


class _SynthPulsar(C.Structure):
    _fields_ = [("period", C.c_double), ("dm", C.c_double), ("duty_cycle", C.c_double),
                ("amplitude", C.c_double), ("phase", C.c_double)]


class _SynthDesc(C.Structure):
    _fields_ = [("nchans", C.c_uint64), ("nsamples", C.c_uint64), ("tsamp", C.c_double),
                ("f_low", C.c_double), ("f_high", C.c_double), ("nbits", C.c_int32), ("npulsars", C.c_int32),
                ("seed", C.c_uint64), ("pulsars", C.POINTER(_SynthPulsar)),
                ("narrowband_mask", C.POINTER(C.c_uint8)), ("narrowband_hz", C.c_double),
                ("narrowband_amplitude", C.c_double), ("impulse_hz", C.c_double),
                ("impulse_amplitude", C.c_double)]


def synth_generate(obs, t_begin: int = 0, t_end: int | None = None, out: np.ndarray | None = None) -> np.ndarray:
    """Rows [t_begin, t_end) of a gaffa_b200.synth.Observation on the host
    cores (synth_oracle.c): uint8 [time][channel], or packed 2-bit bytes
    [time][channel/4] for 2-bit observations.  Same noise bits as the numpy
    and CUDA generators; lets CPU-only callers build an input without the
    CUDA library."""
    from gaffa_b200 import synth  # numpy only: the channel mask
    t_end = obs.nsamples if t_end is None else t_end
    row = obs.nchans if obs.nbits == 8 else obs.nchans // 4
    if out is None:
        out = np.empty((t_end - t_begin, row), np.uint8)
    if out.shape != (t_end - t_begin, row) or out.dtype != np.uint8 or not out.flags.c_contiguous:
        raise ValueError("out must be a contiguous uint8 array of the requested rows")
    ps = (_SynthPulsar * max(1, len(obs.pulsars)))()
    for i, p in enumerate(obs.pulsars):
        ps[i] = _SynthPulsar(p.period, p.dm, p.duty_cycle, p.amplitude, p.phase)
    mask = None
    if obs.rfi.narrowband_fraction > 0.0:
        mask = np.ascontiguousarray(synth._narrowband_mask(obs).astype(np.uint8))
    d = _SynthDesc(obs.nchans, obs.nsamples, obs.tsamp, obs.f_low, obs.f_high, obs.nbits, len(obs.pulsars),
                   obs.seed, ps, None if mask is None else _ptr(mask, C.c_uint8), obs.rfi.narrowband_hz,
                   obs.rfi.narrowband_amplitude, obs.rfi.impulse_hz, obs.rfi.impulse_amplitude)
    rc = PORT_LIB_HANDLE().gfo_synth_generate(C.byref(d), C.c_uint64(t_begin), C.c_uint64(t_end),
                                              out.ctypes.data_as(C.c_void_p))
    if rc:
        raise OracleError(rc, "gfo_synth_generate: invalid observation or rows")
    return out


def ffa64_task_snr(series: np.ndarray, task, widths) -> tuple[np.ndarray, np.ndarray]:
    """FP64 S/N and first best phase, [rows_eval][len(widths)], of one plan task
    (TASK_DTYPE record) on a normalised float series (ffa64_oracle.c)."""
    series = np.ascontiguousarray(series, np.float32)
    widths = np.ascontiguousarray(widths, np.uint64)
    t = np.ascontiguousarray(np.array(task, TASK_DTYPE).reshape(1))
    re, nw = int(t["rows_eval"][0]), len(widths)
    snr = np.zeros((re, nw), np.float64)
    phase = np.zeros((re, nw), np.uint64)
    rc = PORT_LIB_HANDLE().gfo64_ffa_task_snr(
        _ptr(series, C.c_float), C.c_uint64(len(series)), t.ctypes.data_as(C.c_void_p),
        _ptr(widths, C.c_uint64), C.c_uint64(nw), _ptr(snr, C.c_double), _ptr(phase, C.c_uint64))
    if rc:
        raise OracleError(rc, "gfo64_ffa_task_snr: invalid task, widths or series")
    return snr, phase


def ffa64_transform(x: np.ndarray, bins: int) -> np.ndarray:
    """FP64 FFA transform of a [rows][bins] block (ffa64_oracle.c)."""
    x = np.ascontiguousarray(x, np.float64).reshape(-1, bins)
    out = np.zeros_like(x)
    rc = PORT_LIB_HANDLE().gfo64_ffa_transform(_ptr(x, C.c_double), C.c_uint64(x.shape[0]), C.c_uint64(bins),
                                               _ptr(out, C.c_double))
    if rc:
        raise OracleError(rc, "gfo64_ffa_transform: invalid shape")
    return out
