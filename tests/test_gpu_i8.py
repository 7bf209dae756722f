"""The mixed plans' M2L on the fifth-generation tensor cores (csrc/m2l_i8.cu:
dense per-offset operators in four 8-bit slices, exact int32 sums in tensor
memory): against the FP64 path at every order it takes (2..12), for scalar
and vector charges, potential or field alone, adaptive and deep trees; bit
for bit repeatable; and distinct from the rotation M2L that sharded plans,
orders above 12 and SFMM_M2L_KERNEL=rotation use.  Bound: 5e-7 relative L2
against the FP64 path (measured 0.5-2.5e-7), five times under the mixed
form's 1e-6."""
import os

import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_l2
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 5e-7


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


def _eval(t, p, Q, prec, qdim=1, pot=True, field=True):
    npts = Q.shape[0]
    P = np.zeros((npts,) if qdim == 1 else (npts, qdim)) if pot else None
    F = np.zeros((npts, 3)) if field else None
    sf.Plan(t, p, qdim, precision=prec).evaluate(Q, P, F)
    return P, F


@pytest.mark.parametrize("p", [2, 3, 5, 8, 11, 12])
def test_i8_matches_fp64_each_order(ctx, p):
    n = 60_000
    pos, q = W.points("plummer", n, 100 + p), W.charges(n, 100 + p)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    mp, mf = _eval(t, p, q, "mixed")
    fp, ff = _eval(t, p, q, "fp64")
    assert rel_l2(mp, fp) < TOL
    assert rel_l2(mf, ff) < TOL


def test_i8_vector_charges(ctx):
    n = 40_000
    pos = W.points("uniform", n, 31)
    Q = np.random.default_rng(31).uniform(-1, 1, (n, 3))
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    mp, mf = _eval(t, 10, Q, "mixed", qdim=3)
    fp, ff = _eval(t, 10, Q, "fp64", qdim=3)
    assert rel_l2(mp, fp) < TOL
    assert rel_l2(mf, ff) < TOL


def test_i8_potential_or_field_alone(ctx):
    n = 50_000
    pos, q = W.points("shell", n, 32), W.charges(n, 32)
    t = sf.Tree(pos, 20, 32, ctx=ctx)
    both_p, both_f = _eval(t, 9, q, "mixed")
    only_p, _ = _eval(t, 9, q, "mixed", field=False)
    _, only_f = _eval(t, 9, q, "mixed", pot=False)
    assert rel_l2(only_p, both_p) < 1e-13
    assert rel_l2(only_f, both_f) < 1e-13


def test_i8_deep_adaptive_tree(ctx):
    rng = np.random.default_rng(33)
    pos = np.vstack([0.37 + 1e-5 * rng.random((20_000, 3)), rng.random((20_000, 3))])
    q = W.charges(len(pos), 33)
    t = sf.Tree(pos, 20, 32, ctx=ctx)
    assert t.depth >= 14
    mp, mf = _eval(t, 8, q, "mixed")
    fp, ff = _eval(t, 8, q, "fp64")
    assert rel_l2(mp, fp) < TOL
    assert rel_l2(mf, ff) < TOL


def test_i8_repeatable_bit_for_bit(ctx):
    n = 80_000
    pos, q = W.points("gauss2", n, 34), W.charges(n, 34)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    pl = sf.Plan(t, 10, 1, precision="mixed")
    outs = []
    for _ in range(3):
        P, F = np.zeros(n), np.zeros((n, 3))
        pl.evaluate(q, P, F)
        outs.append((P, F))
    for P, F in outs[1:]:
        assert np.array_equal(P, outs[0][0]) and np.array_equal(F, outs[0][1])


def test_i8_differs_from_rotation_path(ctx, monkeypatch):
    """The default mixed plan takes the tensor-core M2L (its rounding differs
    from the rotation kernel's); p = 13 and SFMM_M2L_KERNEL=rotation take the
    rotation M2L; all agree with the FP64 path."""
    n = 50_000
    pos, q = W.points("uniform", n, 35), W.charges(n, 35)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    fp, _ = _eval(t, 12, q, "fp64")
    i8, _ = _eval(t, 12, q, "mixed")
    monkeypatch.setenv("SFMM_M2L_KERNEL", "rotation")
    rot, _ = _eval(t, 12, q, "mixed")
    rot13_env, _ = _eval(t, 13, q, "mixed")
    monkeypatch.delenv("SFMM_M2L_KERNEL")
    rot13, _ = _eval(t, 13, q, "mixed")
    assert not np.array_equal(i8, rot)
    assert np.array_equal(rot13, rot13_env)
    assert rel_l2(i8, fp) < TOL and rel_l2(rot, fp) < 1e-6


def test_i8_against_direct_sum_at_order_12(ctx):
    n = 1_000_000
    pos, q = W.points("uniform", n, 36), W.charges(n, 36)
    t = sf.Tree(pos, 20, 128, ctx=ctx)
    P, F = _eval(t, 12, q, "mixed")
    fP, fF = _eval(t, 12, q, "fp64")
    tg = np.random.default_rng(36).choice(n, 3000, replace=False)
    dp, df = sf.direct(pos, q, tg, ctx=ctx)
    e_mixed, e_fp64 = rel_l2(P[tg], dp), rel_l2(fP[tg], dp)
    assert e_mixed < 1e-6
    assert abs(e_mixed - e_fp64) < 0.05 * e_fp64        # the slices add next to nothing to the truncation error
    assert rel_l2(F[tg], df) < 1e-5
