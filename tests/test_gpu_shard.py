"""The library's sharded evaluation on one device.

A solve split into R shards (fmm_plan_set_shard): R plans of one tree run
the three stages of fmm_evaluate_stage in turn, and between stages the
shards' moments and locals are summed on the device and written back to
every shard -- what an all-reduce over R devices does.  The shards' summed
outputs must equal the unsharded evaluation.  No kernel waits on another
shard: the host orders the stages.  (The same split and stages run over two
gloo ranks on the CPU in test_shard_gloo.py.)
"""
import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import golden_exclusions, golden_tree, load_golden, rel_err_per_target
from oracle import pyoracle
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _sharded(torch, ctx, tree, p, qdim, q_d, R, pot_shape, fld_shape, m2l="rotation", ex=None):
    plans = [sf.Plan(tree, p, qdim).set_m2l(m2l).set_shard(r, R) for r in range(R)]
    if ex is not None:
        for pl in plans:
            pl.set_exclusions(*ex)
    pots = [torch.zeros(pot_shape, dtype=torch.float64, device="cuda") for _ in range(R)]
    flds = [torch.zeros(fld_shape, dtype=torch.float64, device="cuda") if fld_shape else None for _ in range(R)]

    def exchange(which):
        bufs = [pl.exchange_buffer(which) for pl in plans]
        total = torch.stack(bufs).sum(0)
        for b in bufs:
            b.copy_(total)

    for stage in range(3):
        for pl, pot, fld in zip(plans, pots, flds):
            pl.evaluate_stage(q_d, pot, fld, stage)
        torch.cuda.synchronize()
        if stage == 0:
            exchange(0)
        elif stage == 1:
            exchange(1)
            exchange(2)
        torch.cuda.synchronize()
    pot = sum(pots).cpu().numpy()
    fld = sum(flds).cpu().numpy() if fld_shape else None
    return pot, fld


@pytest.fixture(scope="module")
def env():
    torch = pytest.importorskip("torch")
    ctx = sf.Context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    return torch, ctx


@pytest.mark.parametrize("R", [2, 3, 8])
def test_shards_sum_to_the_whole_solve(env, R):
    torch, ctx = env
    n, p = 60_000, 8
    pos, q = W.points("plummer", n, 303), W.charges(n, 303)
    tree = sf.Tree(torch.from_numpy(pos).cuda(), 20, 64, ctx=ctx)
    q_d = torch.from_numpy(q).cuda()
    pot_w = torch.zeros(n, dtype=torch.float64, device="cuda")
    fld_w = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    sf.Plan(tree, p, 1).evaluate(q_d, pot_w, fld_w)
    pot, fld = _sharded(torch, ctx, tree, p, 1, q_d, R, (n,), (n, 3))
    tg = np.arange(0, n, 13)
    sp, sfl = pyoracle.error_scales(pos, q, tg)
    assert rel_err_per_target(pot[tg], pot_w.cpu().numpy()[tg], sp) < TOL
    assert rel_err_per_target(fld[tg], fld_w.cpu().numpy()[tg], sfl) < TOL


@pytest.mark.parametrize("name,m2l", [("vector_n2000_p8_ppn128", "rotation"), ("exclude_n3000_p6", "rotation"),
                                      ("gauss2_n4000_p8", "direct")])
def test_sharded_matches_reference(env, name, m2l):
    """Vector charges (Biot-Savart), exclusions and the direct M2L, split over
    three shards, against the reference's own outputs."""
    torch, ctx = env
    g = load_golden(name)
    n, qdim = g["n"], g["qdim"]
    tree = golden_tree(sf, g, ctx)
    q_d = torch.from_numpy(np.ascontiguousarray(g["q"])).cuda()
    sp, sfl = pyoracle.error_scales(g["pos"], g["q"] if qdim == 1 else np.abs(g["q"]).sum(axis=1))
    if qdim == 1:
        pot, fld = _sharded(torch, ctx, tree, g["p"], 1, q_d, 3, (n,), (n, 3), m2l, golden_exclusions(g))
        assert rel_err_per_target(pot, g["POT"], sp) < TOL
        assert rel_err_per_target(fld, g["FIELD"], sfl) < TOL
    else:
        vp, bi = _sharded(torch, ctx, tree, g["p"], 3, q_d, 3, (n, 3), (n, 3), m2l)
        assert rel_err_per_target(vp, g["VECPOT"], sp) < TOL
        assert rel_err_per_target(bi, g["BIOT"], sfl) < TOL


def test_sharded_plan_refuses_the_one_call_evaluation(env):
    torch, ctx = env
    n = 5000
    pos, q = W.points("uniform", n, 5), W.charges(n, 5)
    tree = sf.Tree(pos, 20, 64, ctx=ctx)
    plan = sf.Plan(tree, 6, 1).set_shard(0, 2)
    with pytest.raises(sf.FMMError):
        plan.evaluate(q, np.zeros(n))
    plan.set_shard(0, 1)                    # back to one shard: evaluate works again
    pot = np.zeros(n)
    plan.evaluate(q, pot)
    assert np.isfinite(pot).all()
