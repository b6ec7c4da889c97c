"""The C ABI from a plain C program: tests/c_abi_check.c compiled with gcc
against include/gaffa_b200.h and linked to libgaffa_b200.so, the way a C or
C++ caller (gaffa's own CUDA API layer) would use it.  Host-only entry points,
so it runs without a GPU; its plan must equal the Python binding's."""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_c_program_builds_plan_and_reports_errors(tmp_path):
    from gaffa_b200 import _lib, core
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not found")
    lib = _lib.LIB_PATH
    if not lib.exists():
        pytest.skip("library not built")
    exe = tmp_path / "c_abi_check"
    subprocess.run([gcc, "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "c_abi_check.c"), "-o", str(exe), str(lib), f"-Wl,-rpath,{lib.parent}"],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    plan = core.make_riptide_ffa_plan(1 << 18, 64e-6, 0.2, 2.0, bins_min=180, bins_max=256)
    m = re.search(r"tasks (\d+) widths (\d+)", out.stdout)
    assert int(m.group(1)) == plan.task_count and int(m.group(2)) == len(plan.width_trials)
    for line in re.findall(r"task .*", out.stdout):
        i, bins, rows, rows_eval, factor = re.match(
            r"task (\d+) bins (\d+) rows (\d+) rows_eval (\d+) factor (\S+)", line).groups()
        t = plan.tasks[int(i)]
        assert (int(bins), int(rows), int(rows_eval)) == (int(t["bins"]), int(t["rows"]), int(t["rows_eval"]))
        assert float(factor) == float(t["downsample_factor"])
    err = re.search(r"error (-?\d+) (.*)", out.stdout)
    assert int(err.group(1)) == _lib.GF_EINVAL and "factor" in err.group(2)


LAYOUTS = {
    # C struct -> ctypes structure or numpy record dtype of gaffa_b200/_lib.py
    "gf_ffa_task": ("FfaTask", "TASK_DTYPE"), "gf_plan_options": ("PlanOptions",),
    "gf_dedisp_desc": ("DedispDesc",), "gf_dedisp_info": ("DedispInfo",),
    "gf_dedisp_batch_item": ("DedispBatchItem",), "gf_filterbank_header": ("FilterbankHeader",),
    "gf_preprocess_desc": ("PreprocessDesc",), "gf_preprocess_info": ("PreprocessInfo",),
    "gf_ffa_info": ("FfaInfo",), "gf_ffa_batch_member": ("FfaBatchMember",),
    "gf_ffa_member_info": ("FfaMemberInfo",), "gf_peak_record": ("PEAK_RECORD_DTYPE",),
    "gf_peak": ("PEAK_DTYPE",), "gf_candidate_options": ("CandidateOptions",), "gf_candidate": ("CAND_DTYPE",),
    "gf_harmonic_context": ("HarmonicContext",), "gf_harmonic_options": ("HarmonicOptions",),
    "gf_harmonic_relation": ("HARMONIC_DTYPE",), "gf_synth_pulsar": ("SynthPulsar",),
    "gf_synth_desc": ("SynthDesc",),
}


def test_binding_struct_layouts_match_the_header(tmp_path):
    """Every POD struct of include/gaffa_b200.h has the size and field offsets
    that the ctypes / numpy declarations of the Python binding assume."""
    import ctypes as C
    from gaffa_b200 import _lib
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not found")
    want, lines = [], []
    for cname, pynames in LAYOUTS.items():
        for pyname in pynames:
            obj = getattr(_lib, pyname)
            if isinstance(obj, type) and issubclass(obj, C.Structure):
                fields = [(f[0], getattr(obj, f[0]).offset) for f in obj._fields_]
                size = C.sizeof(obj)
            else:
                fields = [(n, obj.fields[n][1]) for n in obj.names]
                size = obj.itemsize
            lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
            want.append(f"{cname} size {size}")
            for name, off in fields:
                lines.append(f'  printf("{cname}.{name} %zu\\n", offsetof({cname}, {name}));')
                want.append(f"{cname}.{name} {off}")
    src = tmp_path / "layouts.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "gaffa_b200.h"\nint main(void) {\n' +
                   "\n".join(lines) + "\n  return 0;\n}\n")
    exe = tmp_path / "layouts"
    subprocess.run([gcc, "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    assert [g for g in got if g] == want
