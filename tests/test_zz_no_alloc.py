"""The allocation-free fold entry point, called through the C ABI.

gf_fold_time_series_noalloc exists for callers that cannot allocate device
memory when they fold (their device memory belongs to another allocator's
pool, or cudaMalloc's implicit synchronisation is too costly in their loop).
It must give the same profile and exposure as gf_fold_time_series, call after
call, even though every call reuses one fixed scratch array inside the
library.  This file is collected last so a stop-at-first-failure run has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FOLD_RTOL = 1e-6


def _fold_both(lib, x, is_u32, period, tsamp, nbin, start):
    n = x.numel()
    dev = x.device
    ws = torch.empty(int(lib.gf_fold_workspace_bytes(n, nbin)), dtype=torch.uint8, device=dev)
    p_ref = torch.empty(nbin, dtype=torch.float32, device=dev)
    e_ref = torch.empty(nbin, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.gf_fold_time_series(x.data_ptr(), is_u32, n, period, tsamp, nbin, start, p_ref.data_ptr(),
                                   e_ref.data_ptr(), ws.data_ptr(), stream) == 0
    p = torch.full((nbin,), float("nan"), dtype=torch.float32, device=dev)
    e = torch.full((nbin,), float("nan"), dtype=torch.float64, device=dev)
    status = torch.full((1,), 7, dtype=torch.int32, device=dev)
    rc = lib.gf_fold_time_series_noalloc(x.data_ptr(), is_u32, n, period, tsamp, nbin, start, p.data_ptr(),
                                         e.data_ptr(), status.data_ptr(), stream)
    assert rc == 0, lib.gf_last_error().decode()
    torch.cuda.synchronize()
    return p_ref.cpu().numpy(), e_ref.cpu().numpy(), p.cpu().numpy(), e.cpu().numpy(), int(status.item())


def test_noalloc_fold_matches_allocating_fold_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gaffa_b200 import _lib
    lib = _lib.lib()
    rng = np.random.default_rng(5)
    # first call: a long uint32 series into 64 bins
    x1 = torch.from_numpy(rng.integers(0, 1 << 20, 3_000_000).astype(np.int32)).cuda()
    # second call: a shorter float series into more bins, so stale partial
    # sums left by the first call would show
    x2 = torch.from_numpy(rng.normal(size=200_000).astype(np.float32)).cuda()
    for x, is_u32, period, nbin, start in ((x1, 1, 0.5003, 64, 0), (x2, 0, 0.1234, 250, 17)):
        p_ref, e_ref, p, e, status = _fold_both(lib, x, is_u32, period, 64e-6, nbin, start)
        assert status == 0
        np.testing.assert_allclose(p, p_ref, rtol=FOLD_RTOL, atol=1e-6)
        np.testing.assert_allclose(e, e_ref, rtol=1e-12)


def test_noalloc_fold_matches_reference_fixtures_twice():
    """The reference's own fold_time_series_cpu outputs (tests/golden/ref_small.npz,
    folding.cpp:452-502), two calls in a row through the shared scratch."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pathlib import Path
    from gaffa_b200 import _lib
    lib = _lib.lib()
    g = np.load(Path(__file__).parent / "golden" / "ref_small.npz")
    cases = ((g["fold_in_u32"].view(np.int32), 1, 0.25, 32, 0, g["fold_u32_profile"], g["fold_u32_exposure"]),
             (g["pp_scrunched"].astype(np.float32), 0, 0.1234, 50, 17, g["fold_f32_profile"],
              g["fold_f32_exposure"]))
    for _ in range(2):
        for arr, is_u32, period, nbin, start, want_p, want_e in cases:
            x = torch.from_numpy(np.ascontiguousarray(arr)).cuda()
            _, _, p, e, status = _fold_both(lib, x, is_u32, period, 1e-3, nbin, start)
            assert status == 0
            np.testing.assert_allclose(p, want_p, rtol=FOLD_RTOL, atol=1e-6)
            np.testing.assert_allclose(e, want_e, rtol=1e-12)


def test_noalloc_fold_reports_nonfinite_input_like_the_allocating_fold():
    """A NaN sample sets GF_STATUS_NONFINITE in the caller's status word, as the
    allocating fold sets it in its workspace (the reference rejects such input)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gaffa_b200 import _lib
    lib = _lib.lib()
    x = torch.ones(50_000, dtype=torch.float32, device="cuda")
    x[1234] = float("nan")
    n, nbin = x.numel(), 64
    ws = torch.zeros(int(lib.gf_fold_workspace_bytes(n, nbin)), dtype=torch.uint8, device="cuda")
    p = torch.empty(nbin, dtype=torch.float32, device="cuda")
    e = torch.empty(nbin, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.gf_fold_time_series(x.data_ptr(), 0, n, 0.5, 64e-6, nbin, 0, p.data_ptr(), e.data_ptr(),
                                   ws.data_ptr(), stream) == 0
    off = int(lib.gf_fold_workspace_bytes(n, nbin)) - 16
    alloc_status = int(ws[off:off + 4].cpu().numpy().view(np.uint32)[0])
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.gf_fold_time_series_noalloc(x.data_ptr(), 0, n, 0.5, 64e-6, nbin, 0, p.data_ptr(), e.data_ptr(),
                                           status.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert alloc_status == _lib.STATUS_NONFINITE
    assert int(status.item()) == alloc_status
    # a clean call right after clears the word again
    x[1234] = 0.0
    assert lib.gf_fold_time_series_noalloc(x.data_ptr(), 0, n, 0.5, 64e-6, nbin, 0, p.data_ptr(), e.data_ptr(),
                                           status.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0


def test_noalloc_fold_rejects_work_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gaffa_b200 import _lib
    lib = _lib.lib()
    limit = int(lib.gf_fold_noalloc_max_bytes())
    nbin = 4096
    n = (limit // (2 * nbin * 8) + 1) * 16384  # one block of partials too many
    x = torch.zeros(n, dtype=torch.float32, device="cuda")
    out = torch.empty(nbin, dtype=torch.float32, device="cuda")
    expo = torch.empty(nbin, dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.gf_fold_time_series_noalloc(x.data_ptr(), 0, n, 0.5, 64e-6, nbin, 0, out.data_ptr(), expo.data_ptr(),
                                         status.data_ptr(), None)
    assert rc == _lib.GF_EINVAL
    assert "fixed" in lib.gf_last_error().decode()
    # a length whose scratch size would wrap a 64-bit product is refused too
    huge = (1 << 62) + 16384
    rc = lib.gf_fold_time_series_noalloc(x.data_ptr(), 0, huge, 0.5, 64e-6, 8192, 0, out.data_ptr(),
                                         expo.data_ptr(), status.data_ptr(), None)
    assert rc == _lib.GF_EINVAL
