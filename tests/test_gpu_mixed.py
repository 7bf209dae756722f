"""Mixed-precision form (FP32 near field with two-sum accumulation, 3xTF32
tensor-core M2L): against the FP64 path on the same tree and against the FP64
direct sum.  The stated bound is relative L2 <= 1e-6 against the FP64 path
(the mixed form's own rounding), on top of the truncation error both share."""
import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_l2
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


def _both(ctx, pos, Q, p, qdim=1):
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    n = pos.shape[0]
    shape = (n,) if qdim == 1 else (n, qdim)
    out = {}
    for prec in ("fp64", "mixed"):
        pot, fld = np.zeros(shape), np.zeros((n, 3))
        sf.Plan(t, p, qdim, precision=prec).evaluate(Q, pot, fld)
        out[prec] = (pot, fld)
    return out


@pytest.mark.parametrize("dist,n,p", [("plummer", 200_000, 10), ("uniform", 200_000, 12), ("shell", 100_000, 8),
                                      ("gauss2", 150_000, 6)])
def test_mixed_matches_fp64_path(ctx, dist, n, p):
    pos = W.points(dist, n, 21)
    q = W.charges(n, 21)
    r = _both(ctx, pos, q, p)
    assert np.isfinite(r["mixed"][0]).all() and np.isfinite(r["mixed"][1]).all()
    assert rel_l2(r["mixed"][0], r["fp64"][0]) < MIXED_TOL
    assert rel_l2(r["mixed"][1], r["fp64"][1]) < MIXED_TOL


def test_mixed_vector_charges(ctx):
    n = 100_000
    pos = W.points("uniform", n, 22)
    Q = np.random.default_rng(22).uniform(-1, 1, (n, 3))
    r = _both(ctx, pos, Q, 8, qdim=3)
    assert rel_l2(r["mixed"][0], r["fp64"][0]) < MIXED_TOL
    assert rel_l2(r["mixed"][1], r["fp64"][1]) < MIXED_TOL


def test_mixed_against_direct_sum(ctx):
    n = 1_000_000
    pos = W.points("uniform", n, 23)
    q = W.charges(n, 23)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    pot, fld = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, 12, 1, precision="mixed").evaluate(q, pot, fld)
    tg = np.random.default_rng(23).choice(n, 2000, replace=False)
    dpot, dfld = sf.direct(pos, q, tg, ctx=ctx)
    assert rel_l2(pot[tg], dpot) < 1e-6
    assert rel_l2(fld[tg], dfld) < 1e-5
