"""ctypes binding of libgaffa_b200.so (declarations in include/gaffa_b200.h).

The library is built in-tree (``python -m gaffa_b200.build``).  Loading fails
loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libgaffa_b200.so"

GF_OK = 0
GF_EINVAL = -1
GF_EOVERFLOW = -2
GF_ERUNTIME = -3
GF_ENOMEM = -4
GF_ECUDA = -5
GF_EDATA = -6
GF_EOVERFLOW_PEAKS = -7

STATUS_NONFINITE = 1
STATUS_CONSTANT = 2
STATUS_PEAK_OVERFLOW = 4
STATUS_SCHEDULE = 8

DEDISP_BRUTE = 0
DEDISP_SUBBAND = 1

u64, i32, u32, dbl, vp = C.c_uint64, C.c_int32, C.c_uint32, C.c_double, C.c_void_p


class FfaTask(C.Structure):
    _fields_ = [("downsample_factor", dbl), ("effective_tsamp", dbl), ("input_nsamples", u64),
                ("prepared_nsamples", u64), ("bins", u64), ("rows", u64), ("rows_eval", u64),
                ("period_begin", dbl), ("period_end", dbl)]


class PlanOptions(C.Structure):
    _fields_ = [("period_min", dbl), ("period_max", dbl), ("bins_min", u64), ("bins_max", u64),
                ("min_periods", u64), ("duty_cycle_max", dbl), ("width_trial_spacing", dbl),
                ("max_tasks", u64)]


class DedispDesc(C.Structure):
    _fields_ = [("nsamples", u64), ("nchans", u64), ("frequency_mhz", C.POINTER(dbl)),
                ("dm_low", dbl), ("dm_step", dbl), ("ndm", u64), ("ref_frequency_mhz", dbl),
                ("tsamp", dbl), ("chan_begin", u64), ("chan_end", u64), ("nbits", i32),
                ("algorithm", i32), ("subband_channels", u64), ("ndm_per_nominal", u64),
                ("device_id", i32), ("launch_dms_per_cta", i32), ("launch_chunk_rows", i32),
                ("reserved", i32)]


class DedispInfo(C.Structure):
    _fields_ = [("nout", u64), ("max_delay", i32), ("reserved", i32), ("input_bytes", u64),
                ("staged_bytes", u64), ("staged_row_stride", u64), ("workspace_bytes", u64),
                ("metadata_bytes", u64)]


class PreprocessDesc(C.Structure):
    _fields_ = [("tsamp", dbl), ("window_seconds", dbl), ("min_points", u64), ("normalise", i32),
                ("reject_constant", i32), ("nsamples", u64), ("max_series", u64)]


class PreprocessInfo(C.Structure):
    _fields_ = [("window_samples", u64), ("scrunch_factor", u64), ("low_nsamples", u64),
                ("workspace_bytes", u64)]


class FfaInfo(C.Structure):
    _fields_ = [("ntasks", u64), ("noctaves", u64), ("prepared_floats", u64), ("scratch_bytes", u64),
                ("max_task_elements", u64), ("metadata_bytes", u64), ("nclasses", u64)]


class FfaBatchMember(C.Structure):
    _fields_ = [("tasks", vp), ("ntasks", u64), ("widths", vp), ("nwidths", u64), ("nseries", u64)]


class FfaMemberInfo(C.Structure):
    _fields_ = [("nsamples", u64), ("nseries", u64), ("prepared_floats", u64), ("task_begin", u64),
                ("ntasks", u64), ("noctaves", u64)]


class PreprocessBatchItem(C.Structure):
    _fields_ = [("desc", C.POINTER(PreprocessDesc)), ("dev_series", vp), ("input_is_u32", i32), ("reserved", i32),
                ("nseries", u64), ("stride", u64), ("dev_workspace", vp), ("dev_stats", vp), ("dev_status", vp)]


class DedispBatchItem(C.Structure):
    _fields_ = [("program", vp), ("dev_staged", vp), ("dm_begin", u64), ("dm_count", u64), ("dev_out", vp),
                ("out_stride", u64)]


class CandidateOptions(C.Structure):
    _fields_ = [("frequency_cluster_radius", dbl), ("dm_cluster_radius", u64),
                ("cluster_across_widths", i32), ("reserved", i32), ("max_candidates", u64)]


class HarmonicContext(C.Structure):
    _fields_ = [("observation_seconds", dbl), ("frequency_low_mhz", dbl), ("frequency_high_mhz", dbl)]


class HarmonicOptions(C.Structure):
    _fields_ = [("max_harmonic", u64), ("denominator_max", u64), ("frequency_tolerance_bins", dbl),
                ("phase_distance_max", dbl), ("dm_distance_max", dbl), ("use_snr_consistency", i32),
                ("reserved", i32), ("snr_distance_max", dbl)]


class FilterbankHeader(C.Structure):
    _fields_ = [("header_size", C.c_int64), ("nsamples", C.c_int64)] + \
        [(n, i32) for n in ("telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric", "ibeam",
                            "nbeams", "npuls", "nbins", "nbits", "nifs", "nchans")] + \
        [(n, dbl) for n in ("az_start", "za_start", "src_raj", "src_dej", "tstart", "tsamp", "fch1", "foff",
                            "refdm", "period")] + \
        [("uses_frequency_table", i32), ("reversed", i32), ("rawdatafile", C.c_char * 256),
         ("source_name", C.c_char * 256)]


CHANNEL_ORDER_ASCENDING = 0
CHANNEL_ORDER_FILE = 1


class SynthPulsar(C.Structure):
    _fields_ = [("period", dbl), ("dm", dbl), ("duty_cycle", dbl), ("amplitude", dbl), ("phase", dbl)]


class SynthDesc(C.Structure):
    _fields_ = [("nchans", u64), ("nsamples", u64), ("tsamp", dbl), ("f_low", dbl), ("f_high", dbl),
                ("nbits", i32), ("npulsars", i32), ("seed", u64), ("pulsars", C.POINTER(SynthPulsar)),
                ("narrowband_fraction", dbl), ("narrowband_hz", dbl), ("narrowband_amplitude", dbl),
                ("impulse_hz", dbl), ("impulse_amplitude", dbl), ("narrowband_mask", C.POINTER(C.c_uint8))]


TASK_DTYPE = np.dtype([
    ("downsample_factor", "<f8"), ("effective_tsamp", "<f8"), ("input_nsamples", "<u8"),
    ("prepared_nsamples", "<u8"), ("bins", "<u8"), ("rows", "<u8"), ("rows_eval", "<u8"),
    ("period_begin", "<f8"), ("period_end", "<f8")])
PEAK_RECORD_DTYPE = np.dtype([("series", "<u4"), ("task", "<u4"), ("shift", "<u4"), ("phase", "<u2"),
                              ("width_index", "<u2"), ("snr", "<f4"), ("reserved", "<u4")])
PEAK_DTYPE = np.dtype([
    ("dm", "<f8"), ("dm_index", "<u8"), ("period", "<f8"), ("frequency", "<f8"), ("width", "<u8"),
    ("duty_cycle", "<f8"), ("width_index", "<u8"), ("period_index", "<u8"), ("phase", "<u8"),
    ("shift", "<u8"), ("bins", "<u8"), ("snr", "<f4"), ("reserved", "<u4")])
CAND_DTYPE = np.dtype([
    ("dm", "<f8"), ("dm_index", "<u8"), ("period", "<f8"), ("frequency", "<f8"), ("width", "<u8"),
    ("duty_cycle", "<f8"), ("snr", "<f4"), ("reserved", "<u4"), ("peak_count", "<u8"),
    ("dm_index_min", "<u8"), ("dm_index_max", "<u8"), ("frequency_min", "<f8"),
    ("frequency_max", "<f8"), ("best_peak", PEAK_DTYPE)])

HARMONIC_DTYPE = np.dtype([
    ("is_harmonic", "<i4"), ("reserved", "<i4"), ("parent_index", "<u8"), ("numerator", "<i4"),
    ("denominator", "<i4"), ("frequency_error_bins", "<f8"), ("phase_distance", "<f8"),
    ("dm_distance", "<f8"), ("expected_snr", "<f8"), ("snr_distance", "<f8")])
NO_HARMONIC_PARENT = (1 << 64) - 1

assert C.sizeof(FfaTask) == TASK_DTYPE.itemsize == 72
assert PEAK_RECORD_DTYPE.itemsize == 24 and PEAK_DTYPE.itemsize == 96

class PeakSegment(C.Structure):
    _fields_ = [("record_begin", u64), ("record_count", u64), ("series_offset", u64)]


# (name, restype, argtypes) for every entry point of include/gaffa_b200.h
_SIGNATURES = [
    ("gf_last_error", C.c_char_p, []),
    ("gf_status_string", C.c_char_p, [C.c_int]),
    ("gf_build_info", C.c_char_p, []),
    ("gf_cuda_device_count", C.c_int, [C.POINTER(i32)]),
    ("gf_cuda_runtime_version", C.c_int, [C.POINTER(i32)]),
    ("gf_make_riptide_ffa_plan", C.c_int, [u64, dbl, C.POINTER(PlanOptions), vp, u64, C.POINTER(u64), vp,
                                           u64, C.POINTER(u64)]),
    ("gf_downsampled_size", C.c_int, [u64, dbl, C.POINTER(u64)]),
    ("gf_downsampled_variance", C.c_int, [u64, dbl, C.POINTER(dbl)]),
    ("gf_ffa_task_stdnoise", C.c_int, [C.POINTER(FfaTask), C.POINTER(C.c_float)]),
    ("gf_dedisp_program_create", C.c_int, [C.POINTER(DedispDesc), C.POINTER(vp)]),
    ("gf_dedisp_program_destroy", C.c_int, [vp]),
    ("gf_dedisp_program_info", C.c_int, [vp, C.POINTER(DedispInfo)]),
    ("gf_dedisp_workspace_bytes", C.c_int, [vp, u64, C.POINTER(u64)]),
    ("gf_dedisp_stage", C.c_int, [vp, vp, vp, vp]),
    ("gf_dedisp_stage_from_host", C.c_int, [vp, vp, vp, vp, u64, vp]),
    ("gf_dedisp_run", C.c_int, [vp, vp, u64, u64, vp, u64, vp, vp]),
    ("gf_dedisp_check", C.c_int, [vp, vp]),
    ("gf_preprocess_info_get", C.c_int, [C.POINTER(PreprocessDesc), C.POINTER(PreprocessInfo)]),
    ("gf_preprocess_inplace", C.c_int, [C.POINTER(PreprocessDesc), vp, i32, u64, u64, vp, vp, vp, vp]),
    ("gf_normalise", C.c_int, [vp, u64, u64, u64, vp, vp]),
    ("gf_preprocess_batch_create", C.c_int, [C.POINTER(PreprocessBatchItem), u64, i32, C.POINTER(vp)]),
    ("gf_preprocess_batch_run", C.c_int, [vp, vp]),
    ("gf_preprocess_batch_destroy", C.c_int, [vp]),
    ("gf_ffa_program_create", C.c_int, [vp, u64, vp, u64, u64, i32, C.POINTER(vp)]),
    ("gf_ffa_program_destroy", C.c_int, [vp]),
    ("gf_ffa_program_info", C.c_int, [vp, C.POINTER(FfaInfo)]),
    ("gf_ffa_prepare", C.c_int, [vp, vp, u64, u64, vp, vp, vp]),
    ("gf_ffa_search", C.c_int, [vp, vp, u64, C.c_float, vp, vp, u64, vp, vp]),
    ("gf_ffa_expand_peaks", C.c_int, [vp, vp, u64, u64, dbl, dbl, vp]),
    ("gf_ffa_transform", C.c_int, [vp, u64, u64, vp, vp, vp]),
    ("gf_dedisp_batch_create", C.c_int, [C.POINTER(DedispBatchItem), u64, C.POINTER(vp)]),
    ("gf_dedisp_batch_run", C.c_int, [vp, vp]),
    ("gf_dedisp_batch_destroy", C.c_int, [vp]),
    ("gf_ffa_batch_create", C.c_int, [C.POINTER(FfaBatchMember), u64, i32, C.POINTER(vp)]),
    ("gf_ffa_batch_member_info", C.c_int, [vp, u64, C.POINTER(FfaMemberInfo)]),
    ("gf_ffa_batch_bind", C.c_int, [vp, C.POINTER(vp)]),
    ("gf_ffa_batch_prepare", C.c_int, [vp, u64, vp, u64, vp, vp]),
    ("gf_ffa_batch_bind_series", C.c_int, [vp, C.POINTER(vp), C.POINTER(u64), C.POINTER(vp)]),
    ("gf_ffa_batch_prepare_all", C.c_int, [vp, vp]),
    ("gf_ffa_batch_search", C.c_int, [vp, C.c_float, vp, vp, u64, vp, vp]),
    ("gf_ffa_batch_expand_peaks", C.c_int, [vp, vp, u64, vp, vp, vp, vp, vp]),
    ("gf_sort_peaks", C.c_int, [vp, u64]),
    ("gf_select_candidates", C.c_int, [vp, u64, dbl, C.POINTER(CandidateOptions), vp, u64, C.POINTER(u64)]),
    ("gf_select_candidates_device_workspace", C.c_int, [u64, C.POINTER(u64)]),
    ("gf_select_candidates_device", C.c_int, [vp, vp, C.POINTER(PeakSegment), u64, dbl, dbl, dbl,
                                              C.POINTER(CandidateOptions), vp, u64, vp, u64, C.POINTER(u64), vp]),
    ("gf_fold_workspace_bytes", u64, [u64, u64]),
    ("gf_fold_time_series", C.c_int, [vp, i32, u64, dbl, dbl, u64, u64, vp, vp, vp, vp]),
    ("gf_synth_generate", C.c_int, [C.POINTER(SynthDesc), u64, u64, vp, vp]),
    ("gf_fold_noalloc_max_bytes", u64, []),
    ("gf_fold_time_series_noalloc", C.c_int, [vp, i32, u64, dbl, dbl, u64, u64, vp, vp, vp, vp]),
    ("gf_dedisperse_spectrum", C.c_int, [vp, i32, u64, u64, C.POINTER(dbl), dbl, dbl, dbl, u64, u64, vp,
                                         C.POINTER(u64), vp]),
    ("gf_filterbank_read_header", C.c_int, [C.c_char_p, i32, C.POINTER(FilterbankHeader), vp, u64]),
    ("gf_filterbank_read_host", C.c_int, [C.c_char_p, i32, u64, u64, vp]),
    ("gf_filterbank_load", C.c_int, [C.c_char_p, i32, u64, u64, vp, vp, u64, vp]),
    ("gf_fold_spectrum", C.c_int, [vp, i32, u64, u64, dbl, dbl, u64, u64, u64, u64, vp, vp, vp, vp]),
    ("gf_project_folded_cube", C.c_int, [vp, vp, u64, u64, u64, vp, vp, vp, vp]),
    ("gf_prop_conv_forward", C.c_int, [vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, vp]),
    ("gf_prop_conv_backward", C.c_int, [vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp]),
    ("gf_prop_head", C.c_int, [vp, vp, vp, i32, i32, i32, i32, vp, C.c_float, vp, vp, vp, vp, vp, vp]),
    ("gf_prop_adam", C.c_int, [vp, vp, vp, vp, vp, u64, C.c_float, C.c_float, C.c_float, C.c_float, i32,
                               C.c_float, vp]),
    ("gf_prop_features", C.c_int, [vp, u64, u64, dbl, vp, i32, vp, vp]),
    ("gf_prop_downsample", C.c_int, [vp, u64, u64, i32, u64, vp, u64, vp]),
    ("gf_flag_harmonics", C.c_int, [vp, u64, C.POINTER(HarmonicContext), C.POINTER(HarmonicOptions), vp, vp]),
    ("gf_flag_harmonics_device", C.c_int, [vp, u64, C.POINTER(HarmonicContext), C.POINTER(HarmonicOptions), vp,
                                           vp, i32, vp]),
    ("gf_remove_harmonics", C.c_int, [vp, vp, u64, u64, vp, C.POINTER(u64)]),
]

ENTRY_POINTS = [name for name, _, _ in _SIGNATURES]

_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library with `python -m gaffa_b200.build` "
                "(gaffa_b200 has no CPU fallback)")
        handle = C.CDLL(str(LIB_PATH))
        for name, res, args in _SIGNATURES:
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class GaffaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_EXC = {GF_EINVAL: ValueError, GF_EOVERFLOW: OverflowError, GF_ENOMEM: MemoryError}


def check(rc: int) -> None:
    """Raises the Python analogue of the reference's exception for a status."""
    if rc == GF_OK:
        return
    msg = lib().gf_last_error().decode(errors="replace")
    exc = _EXC.get(rc)
    if exc is not None:
        raise exc(msg)
    raise GaffaError(rc, msg)


def ptr(x) -> int:
    """Device/host address of a torch tensor or numpy array (or None -> 0)."""
    if x is None:
        return None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return int(x)
