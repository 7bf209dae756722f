"""The header-only C++ facade compiles (CPU) and runs the reference's example
flow on a GPU (main.cpp:22-111 written against include/simplefmm_b200.hpp)."""
import os
import subprocess
from pathlib import Path

import pytest

from simplefmm_b200 import build as B

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    lib = B.build()
    out = tmp_path_factory.mktemp("facade") / "facade_main"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(ROOT / "tests/native/facade_main.cpp"),
                    f"-L{lib.parent}", "-lsimplefmm_b200", f"-Wl,-rpath,{lib.parent}", "-o", str(out)], check=True)
    return out


def test_facade_compiles(exe):
    assert exe.exists()


@pytest.mark.gpu
def test_facade_runs_reference_example(exe):
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Relative l2 error of potential" in r.stdout
