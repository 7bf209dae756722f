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


@pytest.fixture(scope="module")
def exe_direct(tmp_path_factory):
    """The same program built with the reference's -DFMM_M2L_DIRECT option."""
    lib = B.build()
    out = tmp_path_factory.mktemp("facade_direct") / "facade_main_direct"
    subprocess.run(["g++", "-std=c++17", "-O2", "-DFMM_M2L_DIRECT", f"-I{ROOT / 'include'}",
                    str(ROOT / "tests/native/facade_main.cpp"), f"-L{lib.parent}", "-lsimplefmm_b200",
                    f"-Wl,-rpath,{lib.parent}", "-o", str(out)], check=True)
    return out


def test_facade_compiles(exe, exe_direct):
    assert exe.exists() and exe_direct.exists()


@pytest.mark.gpu
def test_facade_direct_m2l_option_runs_reference_example(exe, exe_direct):
    """-DFMM_M2L_DIRECT (the dense M2L) prints the same errors as the default build."""
    r0 = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    r1 = subprocess.run([str(exe_direct)], capture_output=True, text=True, timeout=1200)
    assert r0.returncode == 0 and r1.returncode == 0, r1.stdout + r1.stderr
    e0 = [float(x.split("=")[1]) for x in r0.stdout.splitlines() if "Relative l2 error" in x]
    e1 = [float(x.split("=")[1]) for x in r1.stdout.splitlines() if "Relative l2 error" in x]
    assert len(e0) == 2 and len(e1) == 2
    for a, b in zip(e0, e1):
        assert abs(a - b) <= 1e-3 * a


@pytest.mark.gpu
def test_facade_runs_reference_example(exe):
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=dict(os.environ))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Relative l2 error of potential" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["exclude_n3000_p6", "exclude_far_n3000_p6"])
def test_facade_exclusion_forms_match_reference(exe, tmp_path, name):
    """FMM3D(partitioner, comm, self_generator) with rinv(Q, U, is_self) and
    rinv(Q, U), potential and field, through the facade: the reference's
    outputs on the same input to 1e-12 (|d|/S per target)."""
    import struct

    import numpy as np

    from conftest import load_golden, rel_err_per_target
    from oracle import pyoracle

    g = load_golden(name)
    n = g["n"]
    s1, s2 = (int(x) for x in g["strides"])
    near_too = int(bool(g["flags"] & 128))
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("<q4i", n, g["max_ppn"], s1, s2, near_too))
        f.write(np.ascontiguousarray(g["pos"], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(g["q"], dtype=np.float64).tobytes())
    r = subprocess.run([str(exe), "exclude", str(fin), str(fout)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(fout, dtype=np.float64)
    pot, field = out[:n], out[n:].reshape(n, 3)
    sp, sfl = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(pot, g["POT"], sp) < 1e-12
    assert rel_err_per_target(field, g["FIELD"], sfl) < 1e-12
