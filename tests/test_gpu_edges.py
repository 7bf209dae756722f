"""Edge cases of the tree and the evaluation, against the restatement (the
reference has no tests of its own; these are the shapes its code allows):
one and two points, a tree held at max_level with leaves above max_ppn,
points stacked in a tiny cluster far from the rest (a deep, narrow tree), a
refused empty input and a refused degenerate (planar) input."""
import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_err_per_target, tree_keys
from oracle import pyoracle
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def ctx():
    return sf.Context(0)


def _compare(ctx, pos, q, p, max_level=20, ppn=64):
    t = sf.Tree(pos, max_level, ppn, ctx=ctx)
    ot = pyoracle.Tree(pos, max_level, ppn)
    d, od = t.dump(), ot.dump()
    assert t.depth == ot.depth
    for k in tree_keys(od):
        assert np.array_equal(d[k], od[k]), k
    n = len(q)
    pot, fld = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, p, 1).evaluate(q, pot, fld)
    opot, ofld = ot.potential_field(p, q)
    if n > 1:
        sp, sfl = pyoracle.error_scales(pos, q)
        assert rel_err_per_target(pot, opot, sp) < TOL
        assert rel_err_per_target(fld, ofld, sfl) < TOL
    return t, pot, fld


def test_single_point_has_no_interactions(ctx):
    pos = np.array([[0.3, 0.2, 0.7]])
    t, pot, fld = _compare(ctx, pos, np.array([1.5]), 6)
    assert t.depth == 0 and pot[0] == 0.0 and np.all(fld == 0.0)


def test_two_points(ctx):
    pos = np.array([[0.0, 0.0, 0.0], [0.3, 0.4, 1.2]])
    q = np.array([2.0, -1.0])
    _, pot, fld = _compare(ctx, pos, q, 4)
    r = np.linalg.norm(pos[0] - pos[1])
    np.testing.assert_allclose(pot, [q[1] / r, q[0] / r], rtol=1e-14)


def test_max_level_caps_a_dense_tree(ctx):
    """max_level 3 with 40,000 Plummer points: leaves at level 3 hold far more
    than max_ppn, as the reference allows (partition.hpp:93-103)."""
    n = 40_000
    pos, q = W.points("plummer", n, 61), W.charges(n, 61)
    t, _, _ = _compare(ctx, pos, q, 8, max_level=3, ppn=16)
    assert t.depth == 3


def test_deep_narrow_tree(ctx):
    """2,000 points in a cluster 1e-4 wide beside 2,000 spread points: the
    cluster's branch is refined ~14 levels below the rest."""
    rng = np.random.default_rng(7)
    pos = np.vstack([0.61 + 1e-4 * rng.random((2000, 3)), rng.random((2000, 3))])
    q = W.charges(len(pos), 7)
    t, _, _ = _compare(ctx, pos, q, 6, ppn=32)
    assert t.depth >= 12


def test_empty_and_planar_inputs_are_refused(ctx):
    with pytest.raises(sf.FMMError) as e:
        sf.Tree(np.zeros((0, 3)), 20, 64, ctx=ctx)
    assert e.value.status == 1                      # FMM_ERR_INVALID_ARGUMENT
    planar = np.random.default_rng(3).random((500, 3))
    planar[:, 2] = 0.25                             # every point on one z plane
    with pytest.raises(sf.FMMError) as e:
        sf.Tree(planar, 20, 64, ctx=ctx)
    assert e.value.status == 5                      # FMM_ERR_DEGENERATE_INPUT (the reference loops forever)
