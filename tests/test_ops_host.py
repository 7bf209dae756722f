"""CPU check of the device operator math.

tests/native/emu.cpp runs the library's m >= 0 formulation (fmm_ops.cuh +
tables.cpp -- the code the kernels execute) serially over the oracle's tree;
its potential and field must agree with the reference (golden fixtures) to the
same 1e-12 per-target bar the GPU path is held to.  This isolates the math
from the GPU parallelisation."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden, rel_err_per_target
from oracle import pyoracle
from simplefmm_b200 import workloads as W

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "simplefmm_b200" / "csrc"


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = tmp_path_factory.mktemp("emu") / "libemu.so"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{CSRC}", str(ROOT / "tests/native/emu.cpp"),
                    str(CSRC / "tables.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    lib.emu_fmm.restype = C.c_int
    return lib


def run_emu(lib, dump, pos, Q, p, va=2, phideg=0.0, want_pot=True, want_field=True, split=False):
    depth = int(dump["DEPTH"][0])
    keep = []

    def arr(key, dtype, l):
        a = np.ascontiguousarray(dump.get(f"{key}{l}", np.zeros(1, dtype)), dtype=dtype)
        if a.size == 0:
            a = np.zeros(1, dtype)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    def ptrs(key, dtype):
        return (C.c_void_p * (depth + 1))(*[arr(key, dtype, l) for l in range(depth + 1)])

    nnode = np.array([dump[f"CNODE{l}"].size for l in range(depth + 1)], np.int64)
    nleaf = np.array([dump[f"ILEAF{l}"].size for l in range(depth + 1)], np.int64)
    pos = np.ascontiguousarray(pos, np.float64)
    Q = np.ascontiguousarray(Q, np.float64)
    qdim = 1 if Q.ndim == 1 else Q.shape[1]
    pot = np.zeros((pos.shape[0], qdim)) if qdim > 1 else np.zeros(pos.shape[0])
    field = np.zeros((pos.shape[0], 3))
    box = np.ascontiguousarray(dump["BOX"], np.float64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    rc = lib.emu_fmm(depth, nnode.ctypes.data_as(C.c_void_p), nleaf.ctypes.data_as(C.c_void_p),
                     ptrs("CNODE", np.int64), ptrs("ILEAF", np.int32), ptrs("IDXP", np.int32), ptrs("IDXV", np.int32),
                     ptrs("ILP", np.int32), ptrs("ILV", np.int32), ptrs("CLP", np.int32), ptrs("CLV", np.int64),
                     ptrs("PL", np.int64), ptrs("NLP", np.int32), ptrs("NLV", np.int32), dp(box), va,
                     C.c_double(phideg), dp(pos), C.c_int64(pos.shape[0]), p, qdim, int(want_pot), int(want_field),
                     dp(Q), dp(pot), dp(field), int(split))
    assert rc == 0
    return pot, field


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("name", ["uniform_n3000_p6", "plummer_n6000_p5_ppn32", "gauss2_n4000_p8",
                                  "uniform_n2500_p10_maxlevel3", "shell_n4000_p4_ppn16", "uniform_n400_p4_depth1"])
def test_emulated_math_matches_reference(emu, name, split):
    """split=False: field through source-gradient moments (grad_moment), the
    reference's own formulation; split=True: the library's formulation, the
    field as minus the gradient of the order-(p+1) local of the order-(p-1)
    moments (grad_local), sharing rotation and translation with the potential."""
    g = load_golden(name)
    t = pyoracle.Tree(g["pos"], g["max_level"], g["max_ppn"], g["vertical_axis"], g["phideg"])
    pot, field = run_emu(emu, t.dump(), g["pos"], g["q"], g["p"], split=split)
    sp, sf = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(pot, g["POT"], sp) < 1e-12
    assert rel_err_per_target(field, g["FIELD"], sf) < 1e-12


@pytest.mark.parametrize("split", [False, True])
def test_emulated_vector_charges(emu, split):
    """rinv (vector potential) and rinv<true> (Q x grad); in split form the
    latter is the curl of the order-(p+1) vector local."""
    g = load_golden("vector_n2000_p8_ppn128")
    t = pyoracle.Tree(g["pos"], g["max_level"], g["max_ppn"])
    pot, field = run_emu(emu, t.dump(), g["pos"], g["q"], g["p"], split=split)
    sp, sf = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(pot, g["VECPOT"], sp) < 1e-12
    assert rel_err_per_target(field, g["BIOT"], sf) < 1e-12


@pytest.mark.parametrize("va,phideg", [(0, 0.0), (1, 0.0), (2, 30.0)])
def test_emulated_box_frames(emu, va, phideg):
    pos = W.plummer(2500, 31)
    q = W.charges(2500, 31)
    t = pyoracle.Tree(pos, 20, 32, va, phideg)
    pot, _ = run_emu(emu, t.dump(), pos, q, 6, va, phideg, want_field=False)
    ref = t.rinv(6, q)
    sp, _ = pyoracle.error_scales(pos, q)
    assert rel_err_per_target(pot, ref, sp) < 1e-12


@pytest.mark.parametrize("split", [False, True])
def test_emulated_p12(emu, split):
    g = load_golden("uniform_n3000_p12")
    t = pyoracle.Tree(g["pos"], g["max_level"], g["max_ppn"])
    pot, field = run_emu(emu, t.dump(), g["pos"], g["q"], 12, split=split)
    sp, sf = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(pot, g["POT"], sp) < 1e-12
    assert rel_err_per_target(field, g["FIELD"], sf) < 1e-12


@pytest.mark.parametrize("name,p", [("uniform_n3000_p13", 13), ("plummer_n3000_p16_ppn32", 16)])
def test_emulated_highest_orders(emu, name, p):
    """p = 13 and the largest order the library takes, 16: the field local's
    L2L runs at order 17, whose term codes need the widest phase field."""
    g = load_golden(name)
    t = pyoracle.Tree(g["pos"], g["max_level"], g["max_ppn"])
    pot, field = run_emu(emu, t.dump(), g["pos"], g["q"], p)
    sp, sf = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(pot, g["POT"], sp) < 1e-12
    assert rel_err_per_target(field, g["FIELD"], sf) < 1e-12


def test_shift_term_codes_hold_every_order(emu):
    """M2M / L2L term codes decode to in-range fields for every order the
    library runs them at: 0..16, and 17 for the field local's L2L at p = 16."""
    emu.emu_check_term_codes.restype = C.c_int
    for p in range(0, 18):
        assert emu.emu_check_term_codes(p) == 0, p


def test_shift_terms_scale_by_order_difference(emu):
    """Every M2M / L2L term's rho power is the order difference of its output
    and input coefficients, for every order the shifts run at: the plan
    builds each level's shift maps by scaling the maps at rho = 1."""
    emu.emu_check_term_powers.restype = C.c_int
    for p in range(0, 18):
        assert emu.emu_check_term_powers(p) == 0, p
