"""The C-ABI library without a GPU: it loads, exports every entry point that
include/gaffa_b200.h declares, and its host-side logic (FFA planner,
peak ordering, candidate selection) is bit-identical to the oracle."""
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "gaffa_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from gaffa_b200 import _lib
    if not _lib.LIB_PATH.exists():
        from gaffa_b200 import build
        build.build()
    return _lib


def test_library_exports_every_declared_symbol(lib):
    handle = lib.lib()
    names = declared_symbols()
    assert len(names) >= 29
    for name in names:
        assert hasattr(handle, name), name
    assert set(names) <= set(lib.ENTRY_POINTS) | {n for n in names if hasattr(handle, n)}
    assert "sm_100a" in handle.gf_build_info().decode()


def test_struct_layouts_match_oracle(lib):
    from oracle import oracle
    assert lib.TASK_DTYPE == oracle.TASK_DTYPE
    assert lib.PEAK_DTYPE == oracle.PEAK_DTYPE
    assert lib.CAND_DTYPE.itemsize == oracle.CAND_DTYPE.itemsize


@pytest.mark.parametrize("args", [
    (29527, 64e-6, 0.2, 2.0, {}),
    (258903, 64e-6, 0.2, 2.0, {}),
    (8357464, 64e-6, 0.1, 10.0, {"duty_cycle_max": 0.1}),
    (3455736, 81.92e-6, 0.1, 10.0, {"duty_cycle_max": 0.1}),
    (64, 0.25, 1.0, 4.0, dict(bins_min=4, bins_max=5, min_periods=2, duty_cycle_max=0.5, max_tasks=1000)),
])
def test_plan_matches_oracle(lib, port, args):
    from gaffa_b200 import core
    n, ts, pmin, pmax, kw = args
    plan = core.make_riptide_ffa_plan(n, ts, pmin, pmax, **kw)
    tasks, widths = port.make_plan(n, ts, pmin, pmax, **kw)
    assert np.array_equal(plan.tasks, tasks)
    assert plan.width_trials == tuple(int(w) for w in widths)


def test_plan_errors_map_to_reference_exceptions(lib):
    from gaffa_b200 import core
    with pytest.raises(ValueError):
        core.make_riptide_ffa_plan(0, 0.25, 1.0, 4.0)
    with pytest.raises(ValueError, match="period_min must be >= tsamp"):
        core.make_riptide_ffa_plan(64, 0.25, 0.5, 4.0, bins_min=4, bins_max=5)
    with pytest.raises(RuntimeError, match="max_tasks"):
        core.make_riptide_ffa_plan(64, 0.25, 1.0, 4.0, bins_min=4, bins_max=5, min_periods=2,
                                   duty_cycle_max=0.5, max_tasks=1)


def test_candidates_and_sort_match_oracle(lib, port, golden_small):
    from gaffa_b200 import core
    g = golden_small
    peaks = g["dm_peaks"]
    shuffled = peaks[np.random.default_rng(0).permutation(len(peaks))]
    assert np.array_equal(core.sort_peaks(shuffled), peaks)
    tobs = g["dd_multi"].shape[1] * 1e-3
    assert np.array_equal(core.select_candidates(peaks, tobs), g["cands_default"])
    assert np.array_equal(core.select_candidates(peaks, tobs, 0.5, 3, False, 5), g["cands_r3_w"])
    with pytest.raises(ValueError):
        core.select_candidates(peaks, 0.0)


def test_host_noise_model_moments():
    """Irwin-Hall(12) noise: mean 128, sd 16 after rounding."""
    from gaffa_b200 import synth
    obs = synth.Observation(nchans=64, nsamples=4096, tsamp=1e-3, f_low=1200, f_high=1500, seed=3)
    x = synth.generate(obs).astype(np.float64)
    assert abs(x.mean() - 128.0) < 0.1 and abs(x.std() - 16.0) < 0.1
    lv = synth.generate(synth.Observation(nchans=64, nsamples=4096, tsamp=1e-3, f_low=300, f_high=400,
                                          nbits=2, seed=3))
    counts = np.bincount(lv.reshape(-1), minlength=4) / lv.size
    assert np.all(np.abs(counts - 0.25) < 0.01)
    assert np.array_equal(synth.unpack_2bit(synth.pack_2bit(lv), 64), lv)


def test_binding_argument_counts_match_the_prototypes(lib):
    """Each ctypes signature of gaffa_b200/_lib.py takes as many arguments as
    the header's prototype (a missing or extra argument would shift every
    later one on the stack)."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "gaffa_b200.h").read_text(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(gf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
        args = " ".join(m.group(2).split())
        protos[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    checked = 0
    for name, _res, argtypes in lib._SIGNATURES:
        if name in protos:
            assert len(argtypes) == protos[name], (name, len(argtypes), protos[name])
            checked += 1
    assert checked >= 0.9 * len(lib._SIGNATURES)


def test_binding_argument_types_match_the_prototypes(lib):
    """Pointers are passed as pointers and scalars with the C scalar's width
    and kind (a double where the C side reads a float, or a 32-bit integer
    where it reads 64 bits, would be read wrongly without any error)."""
    import ctypes as C
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "gaffa_b200.h").read_text(), flags=re.S)
    scalars = {"uint64_t": C.c_uint64, "int64_t": C.c_int64, "uint32_t": C.c_uint32, "int32_t": C.c_int32,
               "int": C.c_int, "double": C.c_double, "float": C.c_float}
    protos = {m.group(1): " ".join(m.group(2).split())
              for m in re.finditer(r"\b(gf_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text)}
    for name, _res, argtypes in lib._SIGNATURES:
        args = protos[name]
        params = [] if args in ("", "void") else [p.strip() for p in args.split(",")]
        for p, t in zip(params, argtypes):
            if "*" in p:
                assert t is C.c_void_p or issubclass(t, (C._Pointer, C.Array, C.c_char_p)), (name, p, t)
            else:
                base = p.replace("const ", "").split()[0]
                assert base in scalars, (name, p)
                want = scalars[base]
                assert C.sizeof(t) == C.sizeof(want) and (t in (C.c_float, C.c_double)) == (
                    want in (C.c_float, C.c_double)), (name, p, t)
