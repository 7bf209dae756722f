"""The CPU restatement (oracle/fmm_oracle.cpp) is pinned against the
reference's own outputs: the committed golden fixtures, and -- where the
compiled reference is present -- live runs of it."""
import numpy as np
import pytest

from conftest import golden_cases, golden_exclusions, load_golden, rel_err_per_target, rel_l2, tree_keys
from oracle import pyoracle, refio
from simplefmm_b200 import workloads as W

CASES = golden_cases()


def _tree(g):
    box = (g["box_corner"], float(g["box_width"][0])) if "box_corner" in g else None
    return pyoracle.Tree(g["pos"], g["max_level"], g["max_ppn"], g["vertical_axis"], g["phideg"], box=box)


@pytest.mark.parametrize("name", CASES)
def test_tree_bit_exact_vs_golden(name):
    g = load_golden(name)
    if "CNODE0" not in g:
        pytest.skip("fixture has no tree dump")
    t = _tree(g)
    d = t.dump()
    assert np.array_equal(d["BOX"], g["BOX"])
    assert t.depth == int(g["DEPTH"][0])
    for k in tree_keys(g):
        assert np.array_equal(d[k], g[k]), k


@pytest.mark.parametrize("name", CASES)
def test_results_vs_golden(name):
    g = load_golden(name)
    t = _tree(g)
    p = g["p"]
    sp, sf = pyoracle.error_scales(g["pos"], g["q"])
    ex = golden_exclusions(g)
    if "POT" in g:
        pot = t.rinv(p, g["q"])
        if ex is not None:
            pyoracle.subtract_exclusions(t, g["pos"], g["q"], *ex, pot=pot)
        assert rel_err_per_target(pot, g["POT"], sp) < 1e-12
    if "FIELD" in g:
        _, E = t.potential_field(p, g["q"])
        if ex is not None:
            pyoracle.subtract_exclusions(t, g["pos"], g["q"], *ex, field=E)
        assert rel_err_per_target(E, g["FIELD"], sf) < 1e-12
    if "VECPOT" in g:
        assert rel_err_per_target(t.rinv(p, g["q"]), g["VECPOT"], sp) < 1e-12
    if "BIOT" in g:
        assert rel_err_per_target(t.rinv(p, g["q"], gradient=True), g["BIOT"], sf) < 1e-12


def test_keys_match_tree_levels():
    """Per-level keys are prefixes of the level-20 key (box.hpp:58-63 truncates
    u * 2^l; scaling by a power of two is exact)."""
    pos = W.plummer(5000, 3)
    k20 = pyoracle.keys(pos, 20)
    for l in (1, 4, 9, 13):
        assert np.array_equal(pyoracle.keys(pos, l), k20 >> (3 * (20 - l)))


def test_fmm_converges_to_direct_sum():
    """FMM error against the FP64 direct sum falls with p (main.cpp:98-111 metric)."""
    pos = W.uniform_cube(4000, 5)
    q = W.charges(4000, 5)
    t = pyoracle.Tree(pos, 20, 64)
    tgt = np.arange(0, 4000, 7)
    ref = pyoracle.direct(pos, q, tgt)
    errs = [rel_l2(t.rinv(p, q)[tgt], ref) for p in (4, 8, 12)]
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-6


def test_scalar_field_from_biot_runs_matches_direct():
    pos = W.plummer(3000, 6)
    q = W.charges(3000, 6)
    t = pyoracle.Tree(pos, 20, 32)
    _, E = t.potential_field(10, q)
    tgt = np.arange(0, 3000, 5)
    ref = pyoracle.direct(pos, q, tgt, mode="field")
    assert rel_l2(E[tgt], ref) < 1e-4


@pytest.mark.skipif(not refio.have_reference(), reason="compiled reference (oracle/_ref) not built")
def test_restatement_vs_live_reference():
    pos = W.two_gaussians(5000, 23)
    q = W.charges(5000, 23, "sign")
    out = refio.run_reference(pos, q, p=7, max_ppn=40, flags=refio.FLAG_TREE | refio.FLAG_POT | refio.FLAG_FIELD)
    t = pyoracle.Tree(pos, 20, 40)
    d = t.dump()
    for k in tree_keys(out):
        assert np.array_equal(d[k], out[k]), k
    pot, E = t.potential_field(7, q)
    sp, sf = pyoracle.error_scales(pos, q)
    assert rel_err_per_target(pot, out["POT"], sp) < 1e-12
    assert rel_err_per_target(E, out["FIELD"], sf) < 1e-12


@pytest.mark.skipif(not refio.have_reference(), reason="compiled reference (oracle/_ref) not built")
def test_reference_ranks_agree():
    """The reference run as 3 shim ranks (like mpirun -n 3) matches 1 rank."""
    pos = W.uniform_cube(3000, 24)
    q = W.charges(3000, 24)
    a = refio.run_reference(pos, q, p=6, flags=refio.FLAG_POT | refio.FLAG_FIELD, ranks=1)
    b = refio.run_reference(pos, q, p=6, flags=refio.FLAG_POT | refio.FLAG_FIELD, ranks=3)
    sp, sf = pyoracle.error_scales(pos, q)
    assert rel_err_per_target(b["POT"], a["POT"], sp) < 1e-12
    assert rel_err_per_target(b["FIELD"], a["FIELD"], sf) < 1e-12
