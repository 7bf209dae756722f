"""Builds ``simplefmm_b200/libsimplefmm_b200.so`` in-tree for sm_100a.

Every CUDA translation unit is compiled with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and linked
into one shared library exposing the C ABI of include/simplefmm_b200.h.
Objects are rebuilt when any source or header under csrc/ or include/ is
newer.  ``python -m simplefmm_b200.build [-v]`` runs it from the shell.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libsimplefmm_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_lib() -> Path:
    return Path(nvcc()).resolve().parent.parent / "lib64"


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.inc")) + list(INCLUDE.glob("*.h"))


def build(verbose: bool = False, extra_flags=None) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr_time = max((h.stat().st_mtime for h in _headers()), default=0)
    base = [nvcc()] + ARCH + NVCC_FLAGS + [f"-I{CSRC}", f"-I{INCLUDE}"] + list(extra_flags or [])
    jobs = []
    for src in _sources():
        obj = BUILD / (src.stem + ".o")
        if not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_time):
            jobs.append(base + ["-c", str(src), "-o", str(obj)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError(f"compile failed: {cmd[-3]}")
        return r.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(run, jobs))
    objs = [BUILD / (s.stem + ".o") for s in _sources()]
    if jobs or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        run([nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] +
            ["-lcudart", "-Xlinker", "-rpath=" + str(cuda_lib())])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
