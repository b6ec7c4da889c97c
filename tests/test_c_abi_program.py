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
