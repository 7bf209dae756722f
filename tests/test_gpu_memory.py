"""Device memory: released blocks of 4 MiB and more are cached by size and
handed to the next request of that size (csrc/memory.cu), on the same stream
or on another one after an event wait.  Repeated solves of one size must give
bit-identical results, also when consecutive trees and plans live on two
contexts (two streams) and so take over each other's blocks."""
import numpy as np
import pytest

import simplefmm_b200 as sf
from simplefmm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _solve(ctx, pos, q, p):
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    pl = sf.Plan(t, p, 1)
    n = pos.shape[0]
    pot, fld = np.zeros(n), np.zeros((n, 3))
    pl.evaluate(q, pot, fld)
    pl.close()
    t.close()
    return pot, fld


def test_repeated_solves_reuse_blocks_bit_identical():
    n = 400_000                      # points, moments and lists are several MiB each
    pos = W.points("plummer", n, 31)
    q = W.charges(n, 31)
    a, b = sf.Context(0), sf.Context(0)
    ref = _solve(a, pos, q, 8)
    assert np.isfinite(ref[0]).all()
    for ctx in (a, b, a, b):
        pot, fld = _solve(ctx, pos, q, 8)
        assert np.array_equal(pot, ref[0])
        assert np.array_equal(fld, ref[1])


def test_blocks_of_other_sizes_after_reuse():
    # sizes that miss the cache between ones that hit it: fresh blocks, correct results
    a = sf.Context(0)
    for n in (300_000, 310_000, 300_000):
        pos = W.points("uniform", n, 32)
        q = W.charges(n, 32)
        pot, _ = _solve(a, pos, q, 6)
        tg = np.random.default_rng(32).choice(n, 500, replace=False)
        dpot, _ = sf.direct(pos, q, tg, ctx=a)
        assert np.linalg.norm(pot[tg] - dpot) / np.linalg.norm(dpot) < 1e-4


@pytest.mark.gpu
def test_work_queued_after_an_evaluation_on_the_caller_stream_sees_the_result():
    """The near field runs on the context's second stream; it joins back into
    the caller's stream before the sums, so a kernel the caller queues on its
    stream right after fmm_evaluate reads the finished result (no host sync)."""
    import torch
    n = 200_000
    pos = W.points("plummer", n, 13)
    q = W.charges(n, 13)
    ctx = sf.Context(0)
    t = sf.Tree(pos, 20, 64, ctx=ctx)
    plan = sf.Plan(t, 8, 1)
    pot_ref, fld_ref = np.zeros(n), np.zeros((n, 3))
    plan.evaluate(q, pot_ref, fld_ref)
    s = torch.cuda.Stream()
    ctx.set_stream(s.cuda_stream)
    with torch.cuda.stream(s):
        qd = torch.tensor(q, device="cuda")
        pot = torch.zeros(n, dtype=torch.float64, device="cuda")
        fld = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    s.synchronize()
    plan.evaluate(qd, pot, fld)
    with torch.cuda.stream(s):
        copy_pot = pot * 1.0
        copy_fld = fld * 1.0
    s.synchronize()
    assert np.array_equal(copy_pot.cpu().numpy(), pot_ref)
    assert np.array_equal(copy_fld.cpu().numpy(), fld_ref)
