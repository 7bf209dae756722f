"""Batched solves (fmm_solve_batch, csrc/forest.cu): several point sets merged
into one forest and evaluated by one plan and one set of launches through a
CUDA graph that the context updates in place.  Each set's result equals the
set solved by a batch of one (bit for bit in FP64, within the mixed form's
own digits otherwise), and the set's own solve (fmm_evaluate of its own tree)
within the rounding of the scaled coordinates; ragged depths, vector charges,
one output alone, the graph reused across batches of one shape."""
import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_l2
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


def _sets(seed, k, nmin=1000, nmax=40_000):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        dist = ["uniform", "plummer", "shell", "gauss2"][i % 4]
        pos = W.points(dist, n, seed + i) * rng.uniform(0.01, 100.0) + rng.uniform(-50, 50, 3)
        out.append((pos, W.charges(n, seed + i)))
    return out


def _alone(ctx, pos, q, p, precision, leaf=64, qdim=1):
    t = sf.Tree(pos, 20, leaf, ctx=ctx)
    n = len(pos)
    P = np.zeros((n,) if qdim == 1 else (n, qdim))
    F = np.zeros((n, 3))
    sf.Plan(t, p, qdim, precision=precision).evaluate(q, P, F)
    return P, F


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_batch_of_one_and_the_own_solve(ctx, precision):
    sets = _sets(50, 9)
    out = sf.solve_batch(sets, 10, precision=precision, ctx=ctx)
    for (pos, q), (P, F) in zip(sets, out):
        (P1, F1), = sf.solve_batch([(pos, q)], 10, precision=precision, ctx=ctx)
        if precision == "fp64":
            assert np.array_equal(P, P1) and np.array_equal(F, F1)
        else:
            assert rel_l2(P, P1) < 1e-12 and rel_l2(F, F1) < 1e-12
        Pa, Fa = _alone(ctx, pos, q, 10, precision)
        tol = 1e-11 if precision == "fp64" else 1e-6         # rounding of the scaled coordinates
        assert rel_l2(P, Pa) < tol and rel_l2(F, Fa) < tol


def test_batch_ragged_depths_vector_charges_and_leaves(ctx):
    rng = np.random.default_rng(51)
    sets = []
    for i, n in enumerate([1, 2, 300, 5000, 60_000]):
        pos = W.points("plummer", n, 60 + i) if n > 2 else rng.random((n, 3))
        sets.append((pos, rng.uniform(-1, 1, (n, 3))))
    leaves = [64, 64, 16, 32, 128]
    out = sf.solve_batch(sets, 8, qdim=3, leaf=leaves, ctx=ctx)
    for (pos, Q), lf, (P, F) in zip(sets, leaves, out):
        Pa, Fa = _alone(ctx, pos, Q, 8, "fp64", leaf=lf, qdim=3)
        if len(pos) == 1:
            assert np.all(P == 0) and np.all(F == 0)
            continue
        assert rel_l2(P, Pa) < 1e-11 and rel_l2(F, Fa) < 1e-11


def test_batch_one_output_and_graph_reuse(ctx):
    sets = _sets(52, 6, 2000, 20_000)
    before = sf.batch_graph_stats(ctx)
    both = sf.solve_batch(sets, 6, ctx=ctx)
    again = sf.solve_batch(_sets(53, 6, 2000, 20_000), 6, ctx=ctx)   # another batch, same launch shape or not
    pot_only = sf.solve_batch(sets, 6, field=False, ctx=ctx)
    for (P, F), (P2, F2) in zip(both, pot_only):
        assert F2 is None and np.array_equal(P, P2)
    third = sf.solve_batch(sets, 6, ctx=ctx)
    for (P, F), (P3, F3) in zip(both, third):
        assert np.array_equal(P, P3) and np.array_equal(F, F3)
    after = sf.batch_graph_stats(ctx)
    assert after["updated"] > before["updated"]       # a graph of this shape was updated in place
    assert len(again) == 6
