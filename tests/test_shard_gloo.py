"""One solve split over two ranks, on the CPU with the gloo backend.

The library's sharded evaluation (fmm_plan_set_shard / fmm_evaluate_stage)
splits a solve as the reference splits it over MPI ranks: leaves per level
balanced by points (balanced_leaf_range, fmm.hpp:503-522), M2L targets by
contiguous ranges (distributed.hpp:14-25), with the moments and the locals
summed across ranks between stages (fmm.hpp:832-859).  Here two processes run
the oracle's restatement of those stages (the same range code,
simplefmm_b200/csrc/shard_ranges.h) and sum with torch.distributed all_reduce
over gloo; the summed result must equal the unsharded solve.  The GPU kernels
of the same stages are checked on one device in test_gpu_shard.py.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    sys.path.insert(0, str(ROOT))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from oracle import pyoracle
    from simplefmm_b200 import workloads as W

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        dist_name, n, p, ppn, ncomp, gradient = case
        pos = W.points(dist_name, n, 41)
        q = W.charges(n, 41) if ncomp == 1 else np.random.default_rng(42).uniform(-1, 1, (n, 3))
        tree = pyoracle.Tree(pos, 20, ppn)
        ev = pyoracle.ShardedEval(tree, p, ncomp, gradient).set_shard(rank, world)
        U = np.zeros((n,) if ncomp == 1 else (n, 3))

        def sum_over_ranks(views):
            for v in views:                       # every level, in the same order on every rank
                dist.all_reduce(torch.from_numpy(v), op=dist.ReduceOp.SUM)

        ev.stage(0, q, U)
        sum_over_ranks(ev.buffers(0))
        ev.stage(1, q, U)
        sum_over_ranks(ev.buffers(1))
        ev.stage(2, q, U)
        sum_over_ranks([U.reshape(-1)])
        if rank == 0:
            np.save(Path(out_dir) / "sharded.npy", U)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", [("plummer", 8000, 8, 32, 1, False), ("uniform", 5000, 6, 64, 3, True)])
def test_two_ranks_equal_the_whole_solve(tmp_path, case):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    from oracle import pyoracle
    from simplefmm_b200 import workloads as W

    mp.spawn(_rank_main, args=(2, _free_port(), case, str(tmp_path)), nprocs=2, join=True)
    got = np.load(tmp_path / "sharded.npy")
    dist_name, n, p, ppn, ncomp, gradient = case
    pos = W.points(dist_name, n, 41)
    q = W.charges(n, 41) if ncomp == 1 else np.random.default_rng(42).uniform(-1, 1, (n, 3))
    ref = pyoracle.Tree(pos, 20, ppn).rinv(p, q, gradient=gradient)
    # each element's contributions come from exactly one rank, the others add zeros
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def test_balanced_leaf_ranges(tmp_path):
    """The split itself (shard_ranges.h, compiled on its own): per level the
    shards' leaf ranges are consecutive, disjoint and cover every leaf, each
    cut is the first leaf whose running point count reaches its share, and a
    shard's points differ from an equal share by less than one leaf."""
    import subprocess

    exe = tmp_path / "shard_ranges_test"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{ROOT / 'simplefmm_b200' / 'csrc'}",
                    str(ROOT / "tests/native/shard_ranges_test.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
    assert "shard ranges ok" in r.stdout
