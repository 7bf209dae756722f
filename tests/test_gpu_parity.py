"""Parity of the CUDA path with the reference.

Trees and lists are compared bit for bit against the reference's own dumps
(tests/golden, generated by tests/golden/make_golden.py from the compiled
reference).  Potentials and fields must agree per target to 1e-12 relative
to the magnitude sum S_i = sum_j |Q_j|/r_ij (potential) or sum_j |Q_j|/r_ij^2
(field): the size of the terms summed at target i, which FP64 rounding is
proportional to.  Every call goes through the C ABI (libsimplefmm_b200.so).
"""
import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import golden_cases, golden_exclusions, golden_tree, load_golden, rel_err_per_target, rel_l2, tree_keys
from oracle import pyoracle
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


@pytest.mark.parametrize("name", golden_cases())
def test_tree_bit_exact(ctx, name):
    g = load_golden(name)
    t = golden_tree(sf, g, ctx)
    d = t.dump()
    assert t.depth == int(g["DEPTH"][0])
    if "CNODE0" not in g:
        return
    assert np.array_equal(d["BOX"], g["BOX"])
    for k in tree_keys(g):
        assert np.array_equal(d[k], g[k]), k


@pytest.mark.parametrize("name", golden_cases())
def test_results_match_reference(ctx, name):
    g = load_golden(name)
    t = golden_tree(sf, g, ctx)
    plan = sf.Plan(t, g["p"], g["qdim"])
    if "m2l_direct" in g:                # the reference built with -DFMM_M2L_DIRECT: the same option here
        plan.set_m2l("direct")
    ex = golden_exclusions(g)
    if ex is not None:
        plan.set_exclusions(*ex)
    sp, sf_ = pyoracle.error_scales(g["pos"], g["q"])
    n = g["n"]
    if g["qdim"] == 1:
        pot = np.zeros(n)
        field = np.zeros((n, 3)) if "FIELD" in g else None
        plan.evaluate(g["q"], pot, field)
        assert rel_err_per_target(pot, g["POT"], sp) < TOL
        if field is not None:
            assert rel_err_per_target(field, g["FIELD"], sf_) < TOL
    else:
        vp = np.zeros((n, 3))
        bi = np.zeros((n, 3))
        plan.rinv(g["q"], vp)
        plan.rinv(g["q"], bi, gradient=True)
        assert rel_err_per_target(vp, g["VECPOT"], sp) < TOL
        assert rel_err_per_target(bi, g["BIOT"], sf_) < TOL


def test_one_pass_equals_separate_calls(ctx):
    g = load_golden("plummer_n6000_p5_ppn32")
    t = sf.Tree(g["pos"], 20, 32, ctx=ctx)
    plan = sf.Plan(t, 5, 1)
    n = g["n"]
    pot, field = np.zeros(n), np.zeros((n, 3))
    plan.evaluate(g["q"], pot, field)
    pot2, field2 = np.zeros(n), np.zeros((n, 3))
    plan.evaluate(g["q"], pot2, None)
    plan.evaluate(g["q"], None, field2)
    assert np.array_equal(pot, pot2)
    assert np.array_equal(field, field2)


def test_outputs_accumulate(ctx):
    """U is accumulated, never overwritten (fmm.hpp:767, 788; main.cpp:57-61)."""
    g = load_golden("uniform_n3000_p6")
    t = sf.Tree(g["pos"], 20, 64, ctx=ctx)
    plan = sf.Plan(t, 6, 1)
    U = np.full(g["n"], 5.0)
    plan.rinv(g["q"], U)
    plan.rinv(g["q"], U)
    sp, _ = pyoracle.error_scales(g["pos"], g["q"])
    assert rel_err_per_target(U - 5.0, 2 * g["POT"], 2 * sp) < TOL


@pytest.mark.parametrize("dist,n,p,ppn", [("plummer", 40000, 10, 64), ("uniform", 50000, 8, 64),
                                          ("gauss2", 20000, 12, 64), ("shell", 30000, 6, 32)])
def test_medium_against_restatement(ctx, dist, n, p, ppn):
    pos = W.points(dist, n, 101)
    q = W.charges(n, 101)
    ot = pyoracle.Tree(pos, 20, ppn)
    t = sf.Tree(pos, 20, ppn, ctx=ctx)
    d, od = t.dump(), ot.dump()
    for k in tree_keys(od):
        assert np.array_equal(d[k], od[k]), k
    pot, field = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, p, 1).evaluate(q, pot, field)
    opot, ofield = ot.potential_field(p, q)
    tg = np.arange(0, n, 37)
    sp, sfl = pyoracle.error_scales(pos, q, tg)
    assert rel_err_per_target(pot[tg], opot[tg], sp) < TOL
    assert rel_err_per_target(field[tg], ofield[tg], sfl) < TOL


def test_leaf_beside_dense_cluster(ctx):
    """Coarse leaves whose near field holds every point of a dense cluster
    (targets x sources far above one work item's share): their near field is
    summed in parts by several warps and reduced in part order.  All targets
    against the restatement, twice (the parts' order is fixed, so the two
    evaluations agree bit for bit), and the mixed form against FP64."""
    rng = np.random.default_rng(5)
    pos = np.vstack([0.5 + 0.01 * rng.random((30000, 3)), rng.random((300, 3))])
    n = pos.shape[0]
    q = W.charges(n, 5)
    ot = pyoracle.Tree(pos, 20, 64)
    d = ot.dump()
    big = 0
    for l in range(ot.depth + 1):
        size = {ll: np.diff(d[f"IDXP{ll}"]) for ll in range(ot.depth + 1)}
        nl = d[f"NLV{l}"].reshape(-1, 2)
        ptr = d[f"NLP{l}"]
        for f in range(len(size[l])):
            ns = sum(int(size[ll][i]) for ll, i in nl[ptr[f]:ptr[f + 1]])
            big += int(size[l][f]) * ns > 131072
    assert big > 0
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    plan = sf.Plan(t, 8, 1)
    pot, field = np.zeros(n), np.zeros((n, 3))
    plan.evaluate(q, pot, field)
    opot, ofield = ot.potential_field(8, q)
    sp, sfl = pyoracle.error_scales(pos, q)
    assert rel_err_per_target(pot, opot, sp) < TOL
    assert rel_err_per_target(field, ofield, sfl) < TOL
    pot2, field2 = np.zeros(n), np.zeros((n, 3))
    plan.evaluate(q, pot2, field2)
    assert np.array_equal(pot, pot2) and np.array_equal(field, field2)
    mpot, mfield = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, 8, 1, precision="mixed").evaluate(q, mpot, mfield)
    assert rel_l2(mpot, pot) < 1e-6
    assert rel_l2(mfield, field) < 1e-6


def test_large_plummer_against_direct_sum(ctx):
    """Configuration-size check: N = 4M Plummer, p = 10, leaf 64, against the
    FP64 direct sum on seeded sample targets (truncation error only)."""
    n = 4_000_000
    pos = W.plummer(n, 7)
    q = W.charges(n, 7)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    pot, field = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, 10, 1).evaluate(q, pot, field)
    tg = np.random.default_rng(7).choice(n, 1000, replace=False)
    dpot = pyoracle.direct(pos, q, tg)
    dfield = pyoracle.direct(pos, q, tg, mode="field")
    assert rel_l2(pot[tg], dpot) < 1e-5
    assert rel_l2(field[tg], dfield) < 1e-4


def test_edge_cases(ctx):
    # one point: nothing to sum
    t = sf.Tree(np.array([[0.1, 0.2, 0.3]]), ctx=ctx)
    U = np.zeros(1)
    sf.Plan(t, 4, 1).rinv(np.array([1.0]), U)
    assert U[0] == 0.0
    # two points: direct only
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 2.0, 2.0]])
    t = sf.Tree(pos, ctx=ctx)
    U = np.zeros(2)
    sf.Plan(t, 4, 1).rinv(np.array([2.0, -1.0]), U)
    assert np.allclose(U, [-1.0 / 3.0, 2.0 / 3.0], rtol=0, atol=1e-15)
    # coplanar vertical extent: the reference would never leave its box loop
    flat = np.random.default_rng(0).random((100, 3))
    flat[:, 2] = 0.5
    with pytest.raises(sf.FMMError) as e:
        sf.Tree(flat, ctx=ctx)
    assert e.value.status == 5
    # max_level caps refinement: leaves may exceed max_particles_per_node
    pos = W.uniform_cube(5000, 3)
    t = sf.Tree(pos, max_level=2, max_particles_per_node=8, ctx=ctx)
    assert t.depth == 2
    ot = pyoracle.Tree(pos, 2, 8)
    d, od = t.dump(), ot.dump()
    for k in tree_keys(od):
        assert np.array_equal(d[k], od[k]), k


def test_invalid_arguments(ctx):
    t = sf.Tree(W.uniform_cube(1000, 1), ctx=ctx)
    with pytest.raises(sf.FMMError) as e:
        sf.Plan(t, 17, 1)
    assert e.value.status == 2
    with pytest.raises(sf.FMMError):
        sf.Plan(t, 8, 4)
    p1 = sf.Plan(t, 4, 1)
    with pytest.raises(sf.FMMError) as e:
        p1.rinv(np.zeros(1000), np.zeros((1000, 3)), gradient=True)
    assert e.value.status == 2


@pytest.mark.parametrize("order", ["ctx-tree-plan", "plan-ctx-tree", "tree-plan-ctx", "ctx-plan-tree"])
def test_handles_destroyed_in_any_order(order):
    """A plan keeps its tree and a tree its context alive (reference counts),
    so bindings that finalize objects in arbitrary order stay safe."""
    import ctypes as C

    L = sf.load_library()
    ctx, tree, plan = C.c_void_p(), C.c_void_p(), C.c_void_p()
    pos = np.ascontiguousarray(W.uniform_cube(5000, 9))
    q = W.charges(5000, 9)
    assert L.fmm_context_create(0, C.byref(ctx)) == 0
    assert L.fmm_tree_build(ctx, C.c_void_p(pos.ctypes.data), 5000, 0, 20, 64, 2, 0.0, C.byref(tree)) == 0
    assert L.fmm_plan_create(tree, 6, 1, 0, C.byref(plan)) == 0
    handles = {"ctx": (L.fmm_context_destroy, ctx), "tree": (L.fmm_tree_destroy, tree), "plan": (L.fmm_plan_destroy, plan)}
    first = order.split("-")[0]
    fn, h = handles.pop(first)
    assert fn(h) == 0
    if first != "plan":
        U = np.zeros(5000)
        assert L.fmm_rinv(plan, C.c_void_p(q.ctypes.data), C.c_void_p(U.ctypes.data), 0, 0) == 0
        assert np.isfinite(U).all() and np.abs(U).max() > 0
    for name in order.split("-")[1:]:
        fn, h = handles[name]
        assert fn(h) == 0


def test_captured_evaluation_replays_like_evaluate():
    """fmm_plan_capture / fmm_plan_replay: the graph of one evaluation, replayed
    with new charges written into the captured array, gives what evaluate gives."""
    torch = pytest.importorskip("torch")
    ctx = sf.Context(0)                                 # its own stream: capturable
    n = 50_000
    pos = W.points("plummer", n, 31)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    plan = sf.Plan(t, 8, 1)
    q_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    pot_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    fld_d = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    plan.capture(q_d, pot_d, fld_d)
    for seed in (32, 33):
        q = W.charges(n, seed)
        q_d.copy_(torch.from_numpy(q))
        pot_d.zero_()
        fld_d.zero_()
        torch.cuda.synchronize()
        plan.replay()
        ctx.synchronize()
        pot, fld = np.zeros(n), np.zeros((n, 3))
        plan.evaluate(q, pot, fld)
        np.testing.assert_array_equal(pot_d.cpu().numpy(), pot)
        np.testing.assert_array_equal(fld_d.cpu().numpy(), fld)


@pytest.mark.parametrize("name", ["uniform_n3000_p6", "gauss2_n4000_p8", "uniform_n3000_p12", "uniform_n3000_p13",
                                  "vector_n2000_p8_ppn128"])
def test_row_owner_m2l_matches_reference(monkeypatch, ctx, name):
    """The row-owner M2L kernel (k_m2l_rows: runs p < 2 and plans whose
    tensor-core kernel does not fit) forced by its test switch: the same
    reference results as the default kernels."""
    monkeypatch.setenv("SFMM_M2L_KERNEL", "rows")
    g = load_golden(name)
    t = golden_tree(sf, g, ctx)
    plan = sf.Plan(t, g["p"], g["qdim"])
    monkeypatch.delenv("SFMM_M2L_KERNEL")
    sp, sf_ = pyoracle.error_scales(g["pos"], g["q"])
    n = g["n"]
    if g["qdim"] == 1:
        pot, field = np.zeros(n), np.zeros((n, 3))
        plan.evaluate(g["q"], pot, field)
        assert rel_err_per_target(pot, g["POT"], sp) < TOL
        assert rel_err_per_target(field, g["FIELD"], sf_) < TOL
    else:
        vp, bi = np.zeros((n, 3)), np.zeros((n, 3))
        plan.rinv(g["q"], vp)
        plan.rinv(g["q"], bi, gradient=True)
        assert rel_err_per_target(vp, g["VECPOT"], sp) < TOL
        assert rel_err_per_target(bi, g["BIOT"], sf_) < TOL


@pytest.mark.parametrize("p", [0, 1])
def test_lowest_orders_against_restatement(ctx, p):
    """p = 0 and 1 (the row-owner M2L kernel's own orders) against the CPU
    restatement, all targets."""
    n = 20000
    pos, q = W.points("plummer", n, 77), W.charges(n, 77)
    t = sf.Tree(pos, 20, 32, ctx=ctx)
    pot, field = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, p, 1).evaluate(q, pot, field)
    ot = pyoracle.Tree(pos, 20, 32)
    opot, ofield = ot.potential_field(p, q)
    sp, sfl = pyoracle.error_scales(pos, q)
    assert rel_err_per_target(pot, opot, sp) < TOL
    assert rel_err_per_target(field, ofield, sfl) < TOL


@pytest.mark.parametrize("name", ["uniform_n3000_p6", "plummer_n6000_p5_ppn32", "gauss2_n4000_p8", "uniform_n3000_p12",
                                  "vector_n2000_p8_ppn128", "exclude_n3000_p6", "plummer_n3000_p16_ppn32",
                                  "direct_plummer_n4000_p8", "direct_vector_n2000_p6"])
def test_direct_m2l_matches_reference(ctx, name):
    """The reference's FMM_M2L_DIRECT formulation (M2Lc_direct, fmm.hpp:592-618):
    the dense M2L reproduces the reference's results to the same 1e-12."""
    g = load_golden(name)
    t = golden_tree(sf, g, ctx)
    plan = sf.Plan(t, g["p"], g["qdim"]).set_m2l("direct")
    ex = golden_exclusions(g)
    if ex is not None:
        plan.set_exclusions(*ex)
    sp, sf_ = pyoracle.error_scales(g["pos"], g["q"])
    n = g["n"]
    if g["qdim"] == 1:
        pot = np.zeros(n)
        field = np.zeros((n, 3)) if "FIELD" in g else None
        plan.evaluate(g["q"], pot, field)
        assert rel_err_per_target(pot, g["POT"], sp) < TOL
        if field is not None:
            assert rel_err_per_target(field, g["FIELD"], sf_) < TOL
    else:
        vp, bi = np.zeros((n, 3)), np.zeros((n, 3))
        plan.rinv(g["q"], vp)
        plan.rinv(g["q"], bi, gradient=True)
        assert rel_err_per_target(vp, g["VECPOT"], sp) < TOL
        assert rel_err_per_target(bi, g["BIOT"], sf_) < TOL


def test_direct_m2l_equals_rotation_on_a_medium_case(ctx):
    """The two M2L formulations on 40,000 Plummer points, p = 10: equal to
    1e-12 per target (they differ in rounding order only)."""
    n = 40_000
    pos, q = W.points("plummer", n, 202), W.charges(n, 202)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    pot_r, fld_r = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, 10, 1).evaluate(q, pot_r, fld_r)
    pot_d, fld_d = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, 10, 1).set_m2l("direct").evaluate(q, pot_d, fld_d)
    tg = np.arange(0, n, 41)
    sp, sfl = pyoracle.error_scales(pos, q, tg)
    assert rel_err_per_target(pot_d[tg], pot_r[tg], sp) < TOL
    assert rel_err_per_target(fld_d[tg], fld_r[tg], sfl) < TOL


@pytest.mark.parametrize("name", golden_cases())
def test_tree_bit_exact_level_launches(monkeypatch, ctx, name):
    """The level-by-level refinement (a launch chain per level; what runs
    where a cooperative launch is not available) forced by its test switch:
    the reference's trees bit for bit, like the single-launch default."""
    monkeypatch.setenv("SFMM_TREE_REFINE", "levels")
    g = load_golden(name)
    t = golden_tree(sf, g, ctx)
    d = t.dump()
    assert t.depth == int(g["DEPTH"][0])
    if "CNODE0" not in g:
        return
    for k in tree_keys(g):
        assert np.array_equal(d[k], g[k]), k


@pytest.mark.parametrize("dist,n,ppn,max_level", [("uniform", 20000, 4, 20), ("plummer", 60000, 1, 20),
                                                  ("gauss2", 30000, 16, 20), ("shell", 40000, 8, 5),
                                                  ("plummer", 5000, 0, 7), ("uniform", 3000, 5000, 20)])
def test_single_launch_refinement_equals_level_launches(monkeypatch, ctx, dist, n, ppn, max_level):
    """The single cooperative launch (node slots grown between launches when
    the first allocation is short: the first four cases need more than n/8
    nodes) gives the level-by-level tree and lists bit for bit, and the same
    potentials."""
    pos = W.points(dist, n, 5)
    q = W.charges(n, 5)
    out = []
    for mode in (None, "levels"):
        if mode:
            monkeypatch.setenv("SFMM_TREE_REFINE", mode)
        t = sf.Tree(pos, max_level, ppn, ctx=ctx)
        d = t.dump()
        pot, fld = np.zeros(n), np.zeros((n, 3))
        sf.Plan(t, 6, 1).evaluate(q, pot, fld)
        out.append((t.depth, d, pot, fld))
    (da, a, pa, fa), (db, b, pb, fb) = out
    assert da == db
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pa, pb) and np.array_equal(fa, fb)


def test_refinement_wait_runs_out_and_reports(monkeypatch, ctx):
    """The single-launch refinement's bounded waits, run out on purpose: with
    its test switch one block waits on a flag that nothing sets, so the other
    blocks' grid-barrier waits end through the abort flag.  The build fails
    with FMM_ERR_TIMEOUT after about two seconds, and the same context then
    builds the tree as before."""
    import time

    pos = W.points("plummer", 20000, 7)
    ref = sf.Tree(pos, 20, 64, ctx=ctx).dump()
    monkeypatch.setenv("SFMM_TREE_TEST_STALL", "1")
    t0 = time.perf_counter()
    with pytest.raises(sf.FMMError) as e:
        sf.Tree(pos, 20, 64, ctx=ctx)
    assert e.value.status == 7                      # FMM_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 30
    monkeypatch.delenv("SFMM_TREE_TEST_STALL")
    d = sf.Tree(pos, 20, 64, ctx=ctx).dump()
    assert d.keys() == ref.keys()
    for k in ref:
        assert np.array_equal(d[k], ref[k]), k


def test_two_component_charges_equal_two_single_solves(ctx):
    """N = 2 charges (potential only, as FMM3D<double, 2>::rinv gives): each
    output component equals the solve of that component's charges alone, to
    FP64 rounding (the M2L tiles group columns differently)."""
    n = 20000
    pos = W.points("plummer", n, 11)
    q2 = np.ascontiguousarray(np.stack([W.charges(n, 11), W.charges(n, 12)], axis=1))
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    u2 = np.zeros((n, 2))
    sf.Plan(t, 8, 2).rinv(q2, u2)
    for b in range(2):
        u1 = np.zeros(n)
        sf.Plan(t, 8, 1).rinv(np.ascontiguousarray(q2[:, b]), u1)
        assert np.max(np.abs(u2[:, b] - u1)) <= 1e-12 * np.max(np.abs(u1)), b
