"""Parity with the live reference at the workloads' own sizes.

The compiled reference (oracle/_ref/ref_driver: the unmodified reference
headers, built by oracle/Makefile, run as one shim rank per host core like
``mpirun -n cores``) solves the same seeded inputs as the library:

  * 100,000 points uniform in the unit cube, p = 8, leaf 64, charges U[-1,1]
    -- the reference's own CPU workload (main.cpp:36-68 at N = 1e5);
  * 200,000 Plummer points (a = 1, r <= 10), p = 10, leaf 64.

Trees and every per-level list must be bit-exact.  Potential and field are
compared at EVERY point by two measures, both reported:
  * |got_i - ref_i| / S_i with S_i = sum_j |Q_j|/r_ij (potential) or
    sum_j |Q_j|/r_ij^2 (field), the size of the terms summed at i: <= 1e-12;
  * the plain relative error |got_i - ref_i| / |ref_i| over the points whose
    value is not a cancellation (|ref_i| >= 1e-3 of the RMS): <= 1e-9, and its
    median is printed.
"""
import os

import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_err_per_target, tree_keys
from oracle import pyoracle, refio
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12
PLAIN_TOL = 1e-9

CASES = [("uniform", 100_000, 8, 64, 31), ("plummer", 200_000, 10, 64, 32)]


def _cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _plain(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    if ref.ndim == 2:
        d, r = np.linalg.norm(got - ref, axis=1), np.linalg.norm(ref, axis=1)
    else:
        d, r = np.abs(got - ref), np.abs(ref)
    keep = r >= 1e-3 * np.sqrt(np.mean(r * r))
    e = d[keep] / r[keep]
    return float(e.max()), float(np.median(e)), int(keep.sum())


@pytest.mark.skipif(not refio.have_reference(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("dist,n,p,ppn,seed", CASES)
def test_full_size_against_live_reference(dist, n, p, ppn, seed):
    pos, q = W.points(dist, n, seed), W.charges(n, seed)
    ref = refio.run_reference(pos, q, p=p, max_level=20, max_ppn=ppn,
                              flags=refio.FLAG_TREE | refio.FLAG_POT | refio.FLAG_FIELD, ranks=_cores(), timeout=1800)
    ctx = sf.Context(0)
    t = sf.Tree(pos, 20, ppn, ctx=ctx)
    assert t.depth == int(ref["DEPTH"][0])
    d = t.dump()
    assert np.array_equal(d["BOX"], ref["BOX"])
    keys = tree_keys(ref)
    assert keys
    for k in keys:
        assert np.array_equal(d[k], ref[k]), k
    pot, field = np.zeros(n), np.zeros((n, 3))
    sf.Plan(t, p, 1).evaluate(q, pot, field)
    sp, sfl = pyoracle.error_scales(pos, q)
    e_pot = rel_err_per_target(pot, ref["POT"], sp)
    e_fld = rel_err_per_target(field, ref["FIELD"], sfl)
    pm, pmed, pk = _plain(pot, ref["POT"])
    fm, fmed, fk = _plain(field, ref["FIELD"])
    print(f"\n{dist} n={n} p={p}: |d|/S pot {e_pot:.2e} field {e_fld:.2e}; plain relative pot max {pm:.2e} "
          f"median {pmed:.2e} ({pk} pts), field max {fm:.2e} median {fmed:.2e} ({fk} pts)")
    assert e_pot < TOL and e_fld < TOL
    assert pm < PLAIN_TOL and fm < PLAIN_TOL
