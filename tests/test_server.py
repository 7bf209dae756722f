"""Serving loop (fmm_server_*): results are the same alone and in the mix,
admission respects the device-memory budget, oversize requests are rejected,
latency statistics are reported."""
import ctypes as C

import numpy as np
import pytest

import simplefmm_b200 as sf
from conftest import rel_l2
from simplefmm_b200 import workloads as W

TOL = 1e-12


def test_server_argument_checks_need_no_device():
    L = sf.load_library()
    h = C.c_void_p()
    assert L.fmm_server_create(0, 0, 1 << 30, C.byref(h)) == 1          # slots must be >= 1
    assert L.fmm_server_create(0, 2, 0, C.byref(h)) == 1                # budget must be > 0
    rid = C.c_int64()
    assert L.fmm_server_submit(None, None, 10, None, 1, 4, 0, 0, None, None, C.byref(rid)) == 1
    assert L.fmm_server_destroy(None) == 0


def _requests(seed, count, nmax):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(nmax))))
        dist = ["uniform", "plummer", "shell"][i % 3]
        p = [6, 10][(i // 3) % 2]
        reqs.append((W.points(dist, n, seed + i), W.charges(n, seed + i), p))
    return reqs


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_same_alone_and_in_the_mix(precision):
    """Each request's result is the same solved alone (one request in the
    server at a time) and in the mix (all submitted at once, small ones
    batched into shared plans and launches): bit for bit.  Against the plain
    solve of its own tree it differs only by the scaling of a batched
    request's coordinates into the unit cube (FP64) or by the mixed form's
    own rounding."""
    reqs = _requests(100, 12, 60_000)
    srv = sf.Server(0, slots=4, memory_budget=8 << 30)
    alone = []
    for pos, q, p in reqs:
        pot, fld, _ = srv.wait(srv.submit(pos, q, p, precision=precision, leaf=64))
        alone.append((pot, fld))
    b0 = srv.batch_stats()
    ids = [srv.submit(pos, q, p, precision=precision, leaf=64) for pos, q, p in reqs]
    for rid, (pot_a, fld_a) in zip(ids, alone):
        pot, fld, lat = srv.wait(rid)
        assert lat > 0
        np.testing.assert_allclose(pot, pot_a, rtol=0, atol=TOL * np.abs(pot_a).max())
        np.testing.assert_allclose(fld, fld_a, rtol=0, atol=TOL * np.abs(fld_a).max())
    b1 = srv.batch_stats()
    assert b1["batched_requests"] - b0["batched_requests"] == len(reqs)
    assert b1["batches"] - b0["batches"] < len(reqs)          # some shared a plan
    st = srv.stats()
    assert st["completed"] == 2 * len(reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    srv.close()
    ctx = sf.Context(0)
    tol = 1e-10 if precision == "fp64" else 1e-6
    for (pos, q, p), (pot_a, fld_a) in zip(reqs, alone):
        t = sf.Tree(pos, 20, 64, ctx=ctx)
        pot, fld = np.zeros(len(q)), np.zeros((len(q), 3))
        sf.Plan(t, p, 1, precision=precision).evaluate(q, pot, fld)
        assert rel_l2(pot_a, pot) < tol and rel_l2(fld_a, fld) < tol


@pytest.mark.gpu
def test_admission_respects_the_memory_budget():
    reqs = _requests(200, 10, 200_000)
    budget = 3 << 29                             # 1.5 GiB: a few of these requests at a time
    srv = sf.Server(0, slots=8, memory_budget=budget)
    ids = [srv.submit(pos, q, p, leaf=64) for pos, q, p in reqs]
    for rid, (pos, q, p) in zip(ids, reqs):
        pot, fld, _ = srv.wait(rid)
        assert np.isfinite(pot).all() and np.isfinite(fld).all()
    st = srv.stats()
    assert st["peak_bytes"] <= budget              # the estimates admitted at once
    assert st["completed"] == len(reqs)
    mem = srv.memory()
    # every request's measured device allocations stayed below its estimate,
    # and what the running requests held at once stayed below the budget
    assert 0 < mem["worst_measured_over_estimate"] <= 1.0
    assert 0 < mem["peak_measured_bytes"] <= budget
    srv.close()


@pytest.mark.gpu
def test_eight_slots_repeat_the_alone_results():
    """Eight requests at a time on eight streams, five rounds: every result
    equals the request's solve alone in a one-slot server (buffers of
    concurrent requests are disjoint; an allocation overrun shows up here as
    a mismatch)."""
    reqs = _requests(200, 10, 200_000)
    srv = sf.Server(0, slots=1, memory_budget=8 << 30)
    alone = [srv.wait(srv.submit(pos, q, p, leaf=64))[:2] for pos, q, p in reqs]
    srv.close()
    for _ in range(5):
        srv = sf.Server(0, slots=8, memory_budget=8 << 30)
        ids = [srv.submit(pos, q, p, leaf=64) for pos, q, p in reqs]
        for rid, (pot_a, fld_a) in zip(ids, alone):
            pot, fld, _ = srv.wait(rid)
            np.testing.assert_allclose(pot, pot_a, rtol=0, atol=TOL * np.abs(pot_a).max())
            np.testing.assert_allclose(fld, fld_a, rtol=0, atol=TOL * np.abs(fld_a).max())
        srv.close()


@pytest.mark.gpu
def test_oversize_request_is_rejected_and_autotuned_requests_are_correct():
    srv = sf.Server(0, slots=2, memory_budget=256 << 20)
    big = W.points("uniform", 2_000_000, 5)
    with pytest.raises(sf.FMMError) as e:
        srv.submit(big, W.charges(2_000_000, 5), 10)
    assert e.value.status == 6                    # FMM_ERR_OVER_BUDGET
    pos = W.points("plummer", 20_000, 6)
    q = W.charges(20_000, 6)
    ids = [srv.submit(pos, q, 8) for _ in range(4)]          # leaf size from the autotuner
    tg = np.arange(0, 20_000, 97)
    dpot, dfld = sf.direct(pos, q, tg)
    for rid in ids:
        pot, fld, _ = srv.wait(rid)
        assert rel_l2(pot[tg], dpot) < 1e-4
        assert rel_l2(fld[tg], dfld) < 1e-3
    srv.close()
