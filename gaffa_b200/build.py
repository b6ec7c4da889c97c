"""Builds libgaffa_b200.so in-tree from gaffa_b200/csrc with nvcc for sm_100a.

Usage: python -m gaffa_b200.build   (or gaffa_b200.build.build())
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgaffa_b200.so"
SOURCES = ["host.cpp", "dedisperse.cu", "preprocess.cu", "ffa.cu", "fold.cu", "synth.cu", "filterbank.cu", "proposal.cu", "candidates.cu", "harmonics.cu"]
# gaffa's C++ API (include/gaffa/*.h) over the C ABI: plain C++20 host code
CXX_SOURCES = ["cxx_api.cpp"]
CXX_FLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", f"-I{ROOT / 'include'}",
             "-I/usr/local/cuda/include"]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
    "--expt-relaxed-constexpr",
    f"-I{ROOT / 'include'}", f"-I{CSRC}",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: Path, obj: Path) -> None:
    if src.name in CXX_SOURCES:
        cmd = [shutil.which("g++") or "g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [_nvcc(), *NVCC_FLAGS, "-x", "cu", "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed for {src.name}:\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in SOURCES + CXX_SOURCES]
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "gaffa_b200.h"] + list((ROOT / "include" / "gaffa").glob("*.h"))
    newest_header = max(h.stat().st_mtime for h in headers)
    jobs = []
    objs = []
    for src in srcs:
        obj = BUILD / (src.name + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header):
            jobs.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as ex:
        for f in [ex.submit(_compile, s, o) for s, o in jobs]:
            f.result()
    if force or jobs or not LIB.exists():
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
               "-o", str(LIB), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
