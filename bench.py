#!/usr/bin/env python
"""Benchmark of the FMM evaluation path on B200.

Workload (one step = one solve): N = 4,000,000 points from a Plummer sphere
(scale radius 1, radii truncated at 10), charges uniform in [-1, 1], expansion
order p = 10, leaf size 64, FP64: tree build + potential and field at every
point.  Metric: points/s = N / (tree build + evaluation time).

  value  inputs already in HBM: positions and charges are device arrays; the
         step (tree build, plan set-up, evaluation) is timed with CUDA events
         on the stream it runs on; L2 is flushed (256 MiB write) between steps.
  e2e    the same step through the C ABI with pinned host arrays: the
         host->device copy of positions and charges (and of the accumulated
         outputs) and the device->host copy of potential and field are inside
         the timed region.
--gpus N runs N independent replicas (one process per GPU, launched by
torch.distributed.run); value = all points / max-over-ranks time.
--impl reference times the reference's own CPU implementation (the compiled
reference headers, run as one shim rank per host core) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "points/sec at stated rel. error vs FP64 direct sum"
N_DEFAULT, P_DEFAULT, LEAF = 4_000_000, 10, 64
SEED = 2024


def f_m2l(p: int) -> int:
    """Algorithmic FLOPs of one M2L pair and component of the reference's
    rotation scheme: 8 n_rot + 4 T_z + 16 (p+1)^2."""
    n_rot = (p + 1) * (2 * p + 1) * (2 * p + 3) // 3
    t_z = sum((p + 1 - abs(k)) ** 2 for k in range(-p, p + 1))
    return 8 * n_rot + 4 * t_z + 16 * (p + 1) ** 2


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """nvidia-smi samples (every 200 ms) while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                                          "200", "-i", str(self.index)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def fp64_peak_tflops(torch) -> float:
    """Measured FP64 dense GEMM rate (cuBLAS DGEMM via torch), best of 3."""
    n = 8192
    a = torch.rand(n, n, dtype=torch.float64, device="cuda")
    b = torch.rand(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


DATA_DESC = {
    "plummer": "synthetic (seeded Plummer sphere, a=1, r<=10; charges U[-1,1])",
    "uniform": "synthetic (seeded uniform unit cube; charges U[-1,1])",
    "shell": "synthetic (seeded thin spherical shell r=1, thickness 0.01; charges U[-1,1])",
    "gauss2": "synthetic (seeded two Gaussian clusters sigma 0.05, centres 0.5 apart, clipped; charges U[-1,1])",
}


def traffic_per_pair():
    """DRAM bytes per M2L pair from the committed ncu summary, if present."""
    f = ROOT / "profiles" / "m2l_fp64_plummer.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_pair:"):
            return float(line.split(":")[1])
    return None


def cpu_baseline(n_sample: int, p: int, steps: int = 1):
    """Reference CPU implementation (compiled reference headers) on a bounded
    sample of the workload, one shim rank per host core."""
    from oracle import refio

    cores = host_cores()
    pos = __import__("simplefmm_b200.workloads", fromlist=["x"]).plummer(n_sample, SEED + 1)
    q = __import__("simplefmm_b200.workloads", fromlist=["x"]).charges(n_sample, SEED + 1)
    kind = "reference"
    if refio.have_reference():
        vals = []
        for _ in range(steps):
            out = refio.run_reference(pos, q, p=p, max_level=20, max_ppn=LEAF,
                                      flags=refio.FLAG_POT | refio.FLAG_FIELD, ranks=cores)
            t = out["T_TREE"] + out["T_CTOR1"] + out["T_POT"] + out["T_CTOR3G"] + out["T_FIELD"]
            vals.append(n_sample / t)
    else:
        from oracle import pyoracle
        kind, cores = "port", 1
        vals = []
        for _ in range(steps):
            t0 = time.perf_counter()
            tr = pyoracle.Tree(pos, 20, LEAF)
            tr.potential_field(p, q)
            vals.append(n_sample / (time.perf_counter() - t0))
    return vals, {"unit": "points/s", "cores": cores, "kind": kind,
                  "sample": f"Plummer N={n_sample} (seed {SEED + 1}), p={p}, leaf {LEAF}, potential + field "
                            f"(tree + FMM3D set-up + rinv, field via two rinv<true> runs)"}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n_sample = args.ref_sample
    vals, info = cpu_baseline(n_sample, args.p, steps=args.warmup + args.steps)
    timed = vals[args.warmup:] or vals
    v = statistics.median(timed)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Plummer sphere, a=1, r<=10; charges U[-1,1])",
            "config": {"workload": f"plummer_p{args.p}_leaf{LEAF}_fp64_potential+field (bounded CPU sample)",
                       "n": n_sample, "p": args.p, "leaf": LEAF},
            "cpu_baseline": dict(info, value=v),
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_bench(args):
    """Serving stream: seeded requests with Poisson arrivals, N log-uniform in
    [1e3, 1e6], uniform / Plummer / thin shell with equal probability, p in
    {6, 10}, charges U[-1,1].  The server (continuous batching under a memory
    budget, autotuned leaf size, the given precision) against the plain FP64
    path solving one request at a time in arrival order.  Latency = completion
    minus arrival."""
    import threading

    import simplefmm_b200 as sf
    from simplefmm_b200 import workloads as W

    rng = np.random.default_rng(SEED + 4)
    k = args.requests
    ns = np.exp(rng.uniform(np.log(1e3), np.log(1e6), k)).astype(np.int64)
    dists = rng.choice(["uniform", "plummer", "shell"], k)
    ps = rng.choice([6, 10], k)
    arrivals = np.cumsum(rng.exponential(1.0 / args.rate, k))
    reqs = [(W.points(str(d), int(n), SEED + 1000 + i), W.charges(int(n), SEED + 1000 + i), int(p))
            for i, (n, d, p) in enumerate(zip(ns, dists, ps))]
    total_points = int(ns.sum())

    def stream_server(precision):
        srv = sf.Server(0, slots=args.slots, memory_budget=args.budget_gib << 30)
        ids = [None] * k
        t0 = time.perf_counter()

        def feeder():
            for i, (pos, q, p) in enumerate(reqs):
                dt = arrivals[i] - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                ids[i] = srv.submit(pos, q, p, precision=precision)

        th = threading.Thread(target=feeder)
        th.start()
        lat = []
        for i in range(k):
            while ids[i] is None:
                time.sleep(0.0005)
            _, _, l_ms = srv.wait(ids[i])
            lat.append(l_ms)
        th.join()
        span = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        return np.array(lat), span, st

    def stream_plain():
        ctx = sf.Context(0)
        t0 = time.perf_counter()
        lat = []
        for i, (pos, q, p) in enumerate(reqs):
            dt = arrivals[i] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            t = sf.Tree(pos, 20, LEAF, ctx=ctx)
            pot, fld = np.zeros(len(q)), np.zeros((len(q), 3))
            sf.Plan(t, p, 1).evaluate(q, pot, fld)
            t.close()
            lat.append((time.perf_counter() - t0 - arrivals[i]) * 1e3)
        return np.array(lat), time.perf_counter() - t0

    # warm-up: one small solve on each path (tables, modules, pools)
    for pos, q, p in reqs[:2]:
        srv = sf.Server(0, slots=1, memory_budget=args.budget_gib << 30)
        srv.wait(srv.submit(pos, q, p, precision=args.precision))
        srv.close()
    lat_s, span_s, st = stream_server(args.precision)
    lat_p, span_p = stream_plain()
    pct = lambda a, q: float(np.percentile(a, q))  # noqa: E731
    line = {
        "metric": "solves/s on a served mixed-size stream (p50/p99 latency beside)", "value": k / span_s,
        "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32 near field, 3xtf32 M2L, f64 moments and sums",
        "data": "synthetic (seeded; Poisson arrivals; N log-uniform [1e3, 1e6]; uniform / Plummer / shell; p in {6, 10})",
        "config": {"workload": f"serving_stream_{k}_requests_rate{args.rate:g}", "requests": k, "rate_per_s": args.rate,
                   "points_total": total_points, "slots": args.slots, "budget_gib": args.budget_gib,
                   "precision": args.precision, "leaf": "autotuned {32, 64, 128}"},
        "latency_ms": {"p50": pct(lat_s, 50), "p99": pct(lat_s, 99), "mean": float(lat_s.mean())},
        "points_per_s": total_points / span_s,
        "server": st,
        "plain_one_at_a_time": {"solves_per_s": k / span_p, "points_per_s": total_points / span_p,
                                "p50_ms": pct(lat_p, 50), "p99_ms": pct(lat_p, 99), "precision": "fp64",
                                "leaf": LEAF},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--p", type=int, default=P_DEFAULT)
    ap.add_argument("--dist", default="plummer")
    ap.add_argument("--ref-sample", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--serve", action="store_true", help="serving-stream benchmark instead of the solve benchmark")
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--rate", type=float, default=100.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--slots", type=int, default=4)
    ap.add_argument("--budget-gib", type=int, default=32)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    if args.serve:
        serve_bench(args)
        return

    import torch
    import torch.distributed as dist

    import simplefmm_b200 as sf
    from simplefmm_b200 import workloads as W

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    n, p = args.n, args.p
    pos_h = W.points(args.dist, n, SEED)
    q_h = W.charges(n, SEED)
    ctx = sf.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    pos_d = torch.from_numpy(pos_h).cuda()
    q_d = torch.from_numpy(q_h).cuda()
    pot_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    fld_d = torch.zeros(n, 3, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    live = []

    def step():
        # one evaluation as a time-stepping caller runs it: release the
        # previous step's tree and plan, build the tree, set up, evaluate
        while live:
            live.pop().close()
        pot_d.zero_()
        fld_d.zero_()
        tree = sf.Tree(pos_d, 20, LEAF, ctx=ctx)
        plan = sf.Plan(tree, p, 1, precision=args.precision)
        plan.evaluate(q_d, pot_d, fld_d)
        live.extend([plan, tree])
        return tree, plan

    for _ in range(args.warmup):
        tree, plan = step()
        flush.zero_()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    times, m2l_ms, phases = [], [], []
    launches0 = sf.launch_count()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            tree, plan = step()
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
            tm = plan.timings()
            m2l_ms.append(tm["m2l_ms"])
            phases.append(tm)
    launches = (sf.launch_count() - launches0) // max(args.steps, 1)
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = n * world * args.steps / (total_ms * 1e-3)

    # accuracy of the last step against the FP64 direct sum on seeded targets
    n_check = min(n, 10_000)
    tg = np.random.default_rng(SEED).choice(n, n_check, replace=False)
    dpot, dfld = sf.direct(pos_h, q_h, tg, ctx=ctx)
    pot_h, fld_h = pot_d.cpu().numpy(), fld_d.cpu().numpy()
    err_pot = float(np.linalg.norm(pot_h[tg] - dpot) / np.linalg.norm(dpot))
    err_fld = float(np.linalg.norm(fld_h[tg] - dfld) / np.linalg.norm(dfld))

    stats = tree.stats()
    K = 4
    flops_launch = stats["ilist_pairs"] * K * f_m2l(p)
    m2l_avg = statistics.mean(m2l_ms)
    achieved = flops_launch / (m2l_avg * 1e-3) / 1e12
    peak = fp64_peak_tflops(torch)
    tpp = traffic_per_pair()

    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        pos_p, q_p = pin(pos_h), pin(q_h)
        pot_p, fld_p = pin(np.zeros(n)), pin(np.zeros((n, 3)))
        ctx2 = sf.Context(local)
        tr = sf.Tree(pos_p, 20, LEAF, ctx=ctx2)
        sf.Plan(tr, p, 1, precision=args.precision).evaluate(q_p, pot_p, fld_p)
        et = []
        for _ in range(args.steps):
            pot_p[:] = 0
            fld_p[:] = 0
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tr.close()
            tr = sf.Tree(pos_p, 20, LEAF, ctx=ctx2)
            sf.Plan(tr, p, 1, precision=args.precision).evaluate(q_p, pot_p, fld_p)
            et.append(time.perf_counter() - t0)
        tr.close()
        e2e = {"value": n * world / statistics.mean(et), "unit": "points/s",
               "h2d_bytes_per_step": int(pos_p.nbytes + q_p.nbytes + pot_p.nbytes + fld_p.nbytes),
               "d2h_bytes_per_step": int(pot_p.nbytes + fld_p.nbytes)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vals, info = cpu_baseline(args.ref_sample, p)
        cpu = dict(info, value=statistics.median(vals))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 near field, 3xtf32 M2L, f64 moments and sums",
            "data": DATA_DESC.get(args.dist, f"synthetic (seeded {args.dist})"),
            "config": {"workload": f"{args.dist}_n{n}_p{p}_leaf{LEAF}_{args.precision}_potential+field", "n": n,
                       "p": p, "leaf": LEAF, "distribution": args.dist, "precision": args.precision,
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MiB write) between timed steps",
                       "depth": tree.depth, **stats},
            "rel_error_vs_direct": {"potential": err_pot, "field": err_fld, "targets": n_check},
            "phases_ms": {k: round(statistics.mean(ph[k] for ph in phases), 3) for k in phases[0]},
            "step_ms": [round(x, 3) for x in times],
            "tree_ms_per_step": [round(ph["tree_ms"], 3) for ph in phases],
            "roofline": {"bound": "fp64", "kernel": "k_m2l", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "peak_source": "FP64 DGEMM (torch float64 matmul 8192^3) measured in this run",
                         "work": f"ilist pairs x 4 components x F(p)={f_m2l(p)} algorithmic FLOPs per launch",
                         "traffic": (tpp * stats["ilist_pairs"]) if tpp else None},
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(launches),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
