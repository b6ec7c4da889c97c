"""gaffa's C++ CUDA API (include/gaffa/*.h, gaffa_b200/csrc/cxx_api.cpp).

* Signature check: cxx_api.cpp defines every function by its qualified name,
  so it only compiles against headers declaring exactly those signatures.
  It is compiled against include/gaffa/ here and, when the reference
  checkout is present, against the reference's own include/gaffa/ headers.
* A C++ caller (tests/cxx_api_check.cpp) is compiled against include/gaffa/
  and linked with libgaffa_b200.so; on a GPU it runs dedispersion (multi-DM,
  device result + copy_to_host, subband, single DM, aligned spectrum), the
  FFA program, run_ffa_batch_cuda and both search_ffa_cuda forms, and its
  outputs are compared with the reference CPU path bit for bit.
"""
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

CUDA_INCLUDE = "/usr/local/cuda/include"
CUDA_LIB = "/usr/local/cuda/lib64"
LIB = ROOT / "gaffa_b200" / "libgaffa_b200.so"
PEAK_ROW = np.dtype([("series", "<u8"), ("period", "<f8"), ("frequency", "<f8"), ("width", "<u8"),
                     ("duty_cycle", "<f8"), ("width_index", "<u8"), ("period_index", "<u8"), ("phase", "<u8"),
                     ("shift", "<u8"), ("bins", "<u8"), ("snr", "<f4"), ("pad", "<u4")])


def _gxx():
    g = shutil.which("g++")
    if g is None:
        pytest.skip("g++ not available")
    return g


def _reference_include() -> Path | None:
    import __graft_entry__
    p = Path(__graft_entry__.REFERENCE_DIR) / "include" / "gaffa"
    return p.parent if (p / "ffa_cuda.h").exists() else None


def test_api_compiles_against_its_own_headers():
    r = subprocess.run([_gxx(), "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", "-Werror",
                        f"-I{ROOT / 'include'}", f"-I{CUDA_INCLUDE}", str(ROOT / "gaffa_b200" / "csrc" / "cxx_api.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_api_definitions_match_the_reference_declarations():
    ref = _reference_include()
    if ref is None:
        pytest.skip("reference checkout not present")
    # the reference's headers first: every qualified definition must match one of its declarations
    r = subprocess.run([_gxx(), "-std=c++20", "-fsyntax-only", f"-I{ref}", f"-I{ROOT / 'include'}",
                        f"-I{CUDA_INCLUDE}", str(ROOT / "gaffa_b200" / "csrc" / "cxx_api.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_library_exports_the_cxx_api():
    if not LIB.exists():
        pytest.skip("library not built")
    out = subprocess.run(["nm", "-DC", "--defined-only", str(LIB)], capture_output=True, text=True).stdout
    for name in ("gaffa::dedisperse_multi_dm_cuda_device(", "gaffa::dedisperse_subband_cuda_device(",
                 "gaffa::dedisperse_single_dm_cuda(", "gaffa::dedisperse_spectrum_cuda(", "gaffa::copy_to_host(",
                 "gaffa::make_riptide_ffa_plan(", "gaffa::CudaFfaProgram::CudaFfaProgram(",
                 "gaffa::run_ffa_batch_cuda(", "gaffa::search_ffa_cuda(", "gaffa::is_better_ffa_peak(",
                 "gaffa::CudaDeviceMemory::CudaDeviceMemory("):
        assert name in out, name


@pytest.fixture(scope="module")
def checker_binary(tmp_path_factory):
    if not LIB.exists():
        pytest.skip("library not built")
    exe = tmp_path_factory.mktemp("cxx") / "cxx_api_check"
    r = subprocess.run([_gxx(), "-std=c++20", "-O1", f"-I{ROOT / 'include'}", f"-I{CUDA_INCLUDE}",
                        str(ROOT / "tests" / "cxx_api_check.cpp"), "-o", str(exe), str(LIB),
                        f"-Wl,-rpath,{LIB.parent}", f"-L{CUDA_LIB}", "-lcudart", f"-Wl,-rpath,{CUDA_LIB}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cxx_caller_builds_and_links(checker_binary):
    assert checker_binary.exists()


@pytest.mark.gpu
def test_cxx_caller_matches_reference_cpu_path(checker_binary, tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle.oracle import TASK_DTYPE, Oracle
    r = subprocess.run([str(checker_binary), str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ref = Oracle("reference" if Oracle.available("reference") else "port")

    def load(name, dtype):
        return np.fromfile(tmp_path / name, dtype=dtype)

    ns, nc = 3000, 64
    x = load("dd_input.u8", np.uint8).reshape(ns, nc)
    freq = load("dd_freq.f64", np.float64)
    want = ref.dedisperse_multi_dm(x, freq, 0.0, 2.0, 16, 1500.0, 1e-3)
    shape = tuple(load("dd_multi_shape.u64", np.uint64))
    assert shape == want.shape
    assert np.array_equal(load("dd_multi.u32", np.uint32).reshape(want.shape), want)
    assert np.array_equal(load("dd_multi_device.u32", np.uint32).reshape(want.shape), want)
    sb = ref.dedisperse_subband(x, freq, 0.0, 2.0, 16, 1500.0, 1e-3, subband_channels=16, ndm_per_nominal=4)
    assert np.array_equal(load("dd_subband.u32", np.uint32).reshape(sb.shape), sb)
    one = ref.dedisperse_multi_dm(x, freq, 10.0, 1.0, 1, 1500.0, 1e-3)
    assert np.array_equal(load("dd_single.u32", np.uint32).reshape(one.shape), one)
    spec = ref.dedisperse_spectrum(x, freq, 10.0, 1500.0, 1e-3)
    assert tuple(load("dd_spectrum_shape.u64", np.uint64)) == (spec.shape[0], 1, spec.shape[1])
    assert np.array_equal(load("dd_spectrum.u8", np.uint8).reshape(spec.shape), spec)
    assert list(load("errors.u64", np.uint64)) == [1, 2, 3]

    n = 20000
    series = load("ffa_series.f32", np.float32).reshape(3, n)
    tasks = load("ffa_tasks.bin", TASK_DTYPE)
    widths = load("ffa_widths.u64", np.uint64)
    want_tasks, want_widths = ref.make_plan(n, 1e-3, 0.2, 1.0, bins_min=60, bins_max=80)
    assert np.array_equal(tasks, want_tasks) and np.array_equal(widths, want_widths)
    batch = load("ffa_batch.bin", PEAK_ROW)
    fields = ["period", "frequency", "width", "duty_cycle", "width_index", "period_index", "phase", "shift",
              "bins", "snr"]
    total = 0
    for s in range(3):
        w = ref.ffa_search(series[s], tasks, widths, snr_threshold=4.0)
        g = batch[batch["series"] == s]
        assert len(g) == len(w) > 0
        for f in fields:
            assert np.array_equal(g[f], w[f]), (s, f)
        total += len(g)
        if s == 1:
            one = load("ffa_search_program.bin", PEAK_ROW)
            for f in fields:
                assert np.array_equal(one[f], w[f])
        if s == 2:
            one = load("ffa_search_oneshot.bin", PEAK_ROW)
            for f in fields:
                assert np.array_equal(one[f], w[f])
    assert len(batch) == total and np.all(np.diff(batch["series"].astype(np.int64)) >= 0)
