"""gaffa's Python API on the B200 path (gaffa_b200.gaffa).

The cases restate the reference package's own tests (tests/test_dedispersion.py,
tests/test_ffa.py, tests/test_pfold.py, tests/test_filterbank_io.py,
tests/test_dedispersed_wrappers.py) with backend="cuda", on a SIGPROC file
written here (descending channel order, like the reference's basetest.fil).
Where the reference compares its CUDA path with its CPU path, the CUDA
results here are compared with the reference CPU implementation (the
oracle), bit for bit for integer sums and FFA peaks; folds to the fold
tolerance of the other tests.  Argument checks run on the CPU; everything
that computes is marked gpu.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from gaffa_b200 import gaffa  # noqa: E402
from gaffa_b200.gaffa import ffa  # noqa: E402
from gaffa_b200.gaffa.dedispersion import (DedispersedResult, DedispersedSpectrum, dedisperse_multi_dm,  # noqa: E402
                                           dedisperse_single_dm, dedisperse_spectrum, dedisperse_subband)
from gaffa_b200.gaffa.io import Filterbank  # noqa: E402
from gaffa_b200.gaffa.pfold import FoldedProfile, FoldResult, fold, fold_profile, fold_spectrum  # noqa: E402

from test_filterbank import write_fil  # noqa: E402

FOLD_RTOL = 1e-6
NCHANS, NSAMPLES, TSAMP = 64, 4096, 2e-3


@pytest.fixture(scope="module")
def fil(tmp_path_factory):
    """8-bit, 64 channels written high frequency first (foff < 0), 4096
    samples of seeded noise with a dispersed pulse train."""
    rng = np.random.default_rng(31)
    x = np.clip(rng.normal(100, 12, size=(NSAMPLES, NCHANS)), 0, 255)
    f_file = 1500.0 - 4.0 * np.arange(NCHANS)               # file order: descending
    d = np.rint(4148.808 * 40.0 * (f_file ** -2 - f_file.max() ** -2) / TSAMP).astype(int)
    for t0 in range(50, NSAMPLES, 97):
        rows = t0 + d
        ok = rows < NSAMPLES
        x[rows[ok], np.arange(NCHANS)[ok]] += 40
    data = np.clip(x, 0, 255).astype(np.uint8)
    p = tmp_path_factory.mktemp("fil") / "test.fil"
    write_fil(p, data, nchans=NCHANS, fch1=1500.0, foff=-4.0, tsamp=TSAMP)
    return p


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _checker():
    from oracle.oracle import Oracle
    return Oracle("reference" if Oracle.available("reference") else "port")


# ---------------------------------------------------------------- io (CPU) --

def test_filterbank_returns_header_and_numpy_data(fil):
    fb = Filterbank(fil)
    assert isinstance(fb, Filterbank)
    assert fb.header.nsamples == NSAMPLES and fb.header.nifs == 1 and fb.header.nchans == NCHANS
    assert fb.data.shape == (fb.header.nsamples, fb.header.nifs, fb.header.nchans)
    assert fb.header.nbits == 8 and fb.data.dtype == np.uint8
    assert fb.shape == fb.data.shape and fb.dtype == fb.data.dtype and fb.nbytes == fb.data.nbytes
    assert fb.header.foff > 0 and fb.header.frequency_table == sorted(fb.header.frequency_table)


def test_filterbank_preserve_file_order(fil):
    fb = Filterbank(fil, channel_order="preserve_file_order")
    assert fb.header.foff < 0
    asc = Filterbank(fil)
    assert np.array_equal(fb.data[:, :, ::-1], asc.data)


def test_filterbank_rejects_unknown_options(fil):
    with pytest.raises(ValueError, match="unknown channel_order"):
        Filterbank(fil, channel_order="bad")
    with pytest.raises(ValueError, match="unknown reverse_backend"):
        Filterbank(fil, reverse_backend="bad")


def test_filterbank_data_lifetime_survives_wrapper_scope(fil):
    data = Filterbank(fil).data
    assert data.shape[0] > 0 and data[0, 0, 0] >= 0


# ------------------------------------------------------ wrappers (CPU) --

def test_dedispersed_result_wraps_uint32_array_without_copy():
    data = np.array([[1, 2, 3, 4]], dtype=np.uint32)
    result = DedispersedResult(data, tsamp=0.25, dm_low=12.5)
    assert result.data is data and np.shares_memory(result.data, data)
    assert result.shape == (1, 4) and result.dtype == data.dtype and result.nbytes == data.nbytes
    assert (result.ndm, result.nsamples, result.tsamp, result.dm_low, result.dm_step) == (1, 4, 0.25, 12.5, 0.0)
    assert result.backend == "external"


def test_dedispersed_result_rejects_inputs_that_would_copy():
    with pytest.raises(TypeError, match="numpy.ndarray"):
        DedispersedResult([[1, 2]], tsamp=1.0)
    with pytest.raises(ValueError, match="C-contiguous"):
        DedispersedResult(np.zeros((2, 4), np.uint32)[:, ::2], tsamp=1.0)
    with pytest.raises(TypeError, match="uint32 or float32"):
        DedispersedResult(np.zeros((1, 4), np.float64), tsamp=1.0)
    with pytest.raises(ValueError, match="dm_low must be finite and non-negative"):
        DedispersedResult(np.zeros((1, 4), np.uint32), tsamp=1.0, dm_low=-1.0)
    with pytest.raises(ValueError, match="dm_step must be finite and non-negative"):
        DedispersedResult(np.zeros((1, 4), np.uint32), tsamp=1.0, dm_step=float("nan"))


def test_dedispersed_spectrum_wraps_array_without_copy():
    data = np.array([[1, 2], [3, 4]], dtype=np.uint8)
    sp = DedispersedSpectrum(data, tsamp=0.25, dm=42.0, chan_begin=10, chan_end=12)
    assert sp.data is data and sp.shape == (2, 2) and sp.nbytes == data.nbytes
    assert (sp.nsamples, sp.nchans, sp.tsamp, sp.dm, sp.chan_begin, sp.chan_end) == (2, 2, 0.25, 42.0, 10, 12)
    with pytest.raises(ValueError, match="chan_end - chan_begin"):
        DedispersedSpectrum(data, tsamp=0.25, chan_begin=0, chan_end=5)


def test_dedispersion_rejects_unknown_and_cpu_backends(fil):
    fb = Filterbank(fil)
    with pytest.raises(ValueError, match="unknown dedispersion backend"):
        dedisperse_single_dm(fb, dm=0.0, backend="bad")
    with pytest.raises(ValueError, match="CUDA path only"):
        dedisperse_multi_dm(fb, dm_low=0.0, dm_step=1.0, ndm=2, backend="cpu")


# ----------------------------------------------------------- ffa (CPU) --

def make_plan(nsamples: int):
    return ffa.make_riptide_plan(nsamples=nsamples, tsamp=1.0, period_min=2.0, period_max=4.0, bins_min=2,
                                 bins_max=2)


def test_make_riptide_plan_exposes_stable_summary():
    plan = make_plan(8)
    assert isinstance(plan, ffa.FfaPlan)
    assert plan.task_count > 0
    assert plan.width_trials == (1,)


def test_ffa_search_rejects_inputs_that_would_copy():
    plan = make_plan(8)
    with pytest.raises(TypeError, match="numpy.ndarray"):
        ffa.ffa_search([0.0] * 8, plan)
    with pytest.raises(TypeError, match="dtype float32"):
        ffa.ffa_search(np.zeros(8, dtype=np.float64), plan)
    with pytest.raises(ValueError, match="1D"):
        ffa.ffa_search(np.zeros((1, 8), dtype=np.float32), plan)
    with pytest.raises(ValueError, match="C-contiguous"):
        ffa.ffa_search(np.zeros(16, dtype=np.float32)[::2], plan)


def test_ffa_search_rejects_plan_length_mismatch_invalid_limit_and_backends():
    series = np.zeros(8, dtype=np.float32)
    with pytest.raises(ValueError, match="input_nsamples"):
        ffa.ffa_search(series, make_plan(9))
    with pytest.raises(ValueError, match="positive or None"):
        ffa.ffa_search(series, make_plan(8), max_peaks=0)
    with pytest.raises(ValueError, match="'cpu' or 'cuda'"):
        ffa.ffa_search(series, make_plan(8), backend="opencl")
    with pytest.raises(ValueError, match="CUDA path only"):
        ffa.ffa_search(series, make_plan(8), backend="cpu")


def test_cuda_runtime_version_is_reported():
    assert gaffa.cuda_runtime_version() >= 12000
    assert gaffa.cuda_device_count() >= 0


# ----------------------------------------------------------------- GPU --

@pytest.mark.gpu
def test_dedisperse_single_and_multi_match_reference(fil):
    _gpu()
    fb = Filterbank(fil)
    ref = _checker()
    freq = np.asarray(fb.header.frequency_table)
    x = fb.data.reshape(NSAMPLES, NCHANS)
    single = dedisperse_single_dm(fb, dm=40.0)
    assert isinstance(single, DedispersedResult) and single.backend == "cuda" and single.ndm == 1
    assert single.data.dtype == np.uint32 and single.dm_step == 0.0
    want = ref.dedisperse_multi_dm(x, freq, 40.0, 1.0, 1, freq.max(), TSAMP)
    assert np.array_equal(single.data, want)
    multi = dedisperse_multi_dm(fb, dm_low=0.0, dm_step=1.0, ndm=3)
    assert multi.shape == (3, multi.nsamples) and multi.nsamples <= NSAMPLES
    for i in range(3):
        s = dedisperse_single_dm(fb, dm=float(i))
        assert s.nsamples >= multi.nsamples
        assert np.array_equal(multi.data[i], s.data[0, : multi.nsamples])
    assert np.array_equal(multi.data, ref.dedisperse_multi_dm(x, freq, 0.0, 1.0, 3, freq.max(), TSAMP))


@pytest.mark.gpu
def test_dedisperse_subband_matches_reference_and_degenerates_to_multi(fil):
    _gpu()
    fb = Filterbank(fil)
    ref = _checker()
    freq = np.asarray(fb.header.frequency_table)
    x = fb.data.reshape(NSAMPLES, NCHANS)
    multi = dedisperse_multi_dm(fb, dm_low=0.0, dm_step=1.0, ndm=4)
    sub1 = dedisperse_subband(fb, dm_low=0.0, dm_step=1.0, ndm=4, subband_channels=1, ndm_per_nominal=1)
    assert sub1.shape == multi.shape and np.array_equal(sub1.data, multi.data)
    sub = dedisperse_subband(fb, dm_low=5.0, dm_step=0.5, ndm=40, subband_channels=16, ndm_per_nominal=8)
    want = ref.dedisperse_subband(x, freq, 5.0, 0.5, 40, freq.max(), TSAMP, subband_channels=16,
                                  ndm_per_nominal=8)
    assert np.array_equal(sub.data, want)


@pytest.mark.gpu
def test_dedisperse_spectrum_matches_reference(fil):
    _gpu()
    fb = Filterbank(fil)
    ref = _checker()
    zero = dedisperse_spectrum(fb, dm=0.0)
    assert isinstance(zero, DedispersedSpectrum) and zero.backend == "cuda"
    assert zero.shape == (NSAMPLES, NCHANS) and zero.dtype == fb.data.dtype
    assert np.array_equal(zero.data, fb.data[:, 0, :])
    sp = dedisperse_spectrum(fb, dm=40.0)
    single = dedisperse_single_dm(fb, dm=40.0)
    assert sp.nsamples == single.nsamples
    assert np.array_equal(sp.data.sum(axis=1, dtype=np.uint32), single.data[0])
    freq = np.asarray(fb.header.frequency_table)
    want = ref.dedisperse_spectrum(fb.data.reshape(NSAMPLES, NCHANS), freq, 40.0, freq.max(), TSAMP)
    assert np.array_equal(sp.data, want)


@pytest.mark.gpu
def test_ffa_search_cuda_returns_the_reference_peaks():
    _gpu()
    series = np.array([0, 0, 0, 5, 0, 0, 0, 5], dtype=np.float32)
    plan = make_plan(series.size)
    peaks = ffa.ffa_search(series, plan, snr_threshold=0.0)
    assert peaks and all(isinstance(p, ffa.FfaPeak) for p in peaks)
    assert all(peaks[i].snr >= peaks[i + 1].snr for i in range(len(peaks) - 1))
    assert peaks[0].period > 0.0 and peaks[0].frequency > 0.0 and peaks[0].width > 0 and peaks[0].bins == 2
    assert ffa.ffa_search(series, plan, snr_threshold=1000.0) == []
    # a realistic plan against the reference CPU search, field by field
    ref = _checker()
    rng = np.random.default_rng(4)
    n = 60_000
    x = rng.normal(size=n).astype(np.float32)
    x[::457] += 3.0
    plan = ffa.make_riptide_plan(nsamples=n, tsamp=1e-3, period_min=0.2, period_max=1.0, bins_min=60,
                                 bins_max=80)
    got = ffa.ffa_search(x, plan, snr_threshold=5.0)
    tasks, widths = ref.make_plan(n, 1e-3, 0.2, 1.0, bins_min=60, bins_max=80)
    want = ref.ffa_search(x, tasks, widths, snr_threshold=5.0)
    assert len(got) == len(want) > 0
    for g, w in zip(got, want):
        assert (g.period, g.frequency, g.snr, g.width, g.duty_cycle, g.phase, g.shift, g.bins, g.width_index,
                g.period_index) == (w["period"], w["frequency"], np.float32(w["snr"]), w["width"],
                                    w["duty_cycle"], w["phase"], w["shift"], w["bins"], w["width_index"],
                                    w["period_index"])
    with pytest.raises(RuntimeError, match="max_peaks"):
        ffa.ffa_search(x, plan, snr_threshold=5.0, max_peaks=1)


@pytest.mark.gpu
def test_fold_profile_and_spectrum_match_reference(fil):
    _gpu()
    fb = Filterbank(fil)
    ref = _checker()
    dd = dedisperse_single_dm(fb, dm=40.0)
    prof = fold_profile(dd, period=97 * TSAMP, nbin=32)
    assert isinstance(prof, FoldedProfile) and prof.profile.shape == (32,) and prof.phase[1] == np.float32(1 / 32)
    want_p, want_e = ref.fold(dd.data[0], 97 * TSAMP, TSAMP, 32)
    np.testing.assert_allclose(prof.profile, want_p, rtol=FOLD_RTOL)
    np.testing.assert_allclose(prof.exposure, want_e, rtol=1e-12)
    wrapped = DedispersedResult(np.array([[1.0, 2.0, 3.0, 4.0]], np.float32), tsamp=1.0)
    np.testing.assert_allclose(fold(wrapped, period=2.0, nbin=2).profile, np.array([2.0, 3.0], np.float32))
    sp = dedisperse_spectrum(fb, dm=40.0)
    res = fold_spectrum(sp, period=97 * TSAMP, nbin=16, tsubint=1.0, nsubband=8)
    assert isinstance(res, FoldResult)
    assert res.cube.shape == (res.nsubint, 8, 16) and res.exposure.shape == (res.nsubint, 16)
    assert res.time.shape == (res.nsubint,) and res.time[0] == pytest.approx(res.tsubint / 2)
    assert isinstance(fold(sp, period=97 * TSAMP, nbin=16, tsubint=1.0), FoldResult)
    if ref.kind != "reference":
        pytest.skip("the spectrum fold is checked against the reference's own sources (oracle/_ref)")
    want = ref.fold_dedispersed_spectrum(sp.data, 97 * TSAMP, TSAMP, 16, tsubint=1.0, output_channels=8)
    np.testing.assert_allclose(res.cube, want["cube"], rtol=FOLD_RTOL, atol=1e-4)
    np.testing.assert_allclose(res.profile, want["profile"], rtol=FOLD_RTOL, atol=1e-4)
