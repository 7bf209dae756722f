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
torch.distributed.run); value = all points / max-over-ranks time.  With
--shard, the N ranks split one solve instead (strong scaling; the moments,
locals and outputs are summed with NCCL all-reduces between the stages).
--impl reference times the reference's own CPU implementation (the compiled
reference headers, run as one shim rank per host core) on a bounded sample of
the same workload: the first 1M of its points.
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
    """The reference's operation count of one M2L pair and charge component
    of its rotation scheme (fmm.hpp:620-688): 8 n_rot + 4 T_z + 16 (p+1)^2.
    The reference runs it for 4 components (potential + two gradient runs of
    3); reported as frac_ref_ops only."""
    n_rot = (p + 1) * (2 * p + 1) * (2 * p + 3) // 3
    t_z = sum((p + 1 - abs(k)) ** 2 for k in range(-p, p + 1))
    return 8 * n_rot + 4 * t_z + 16 * (p + 1) ** 2


def m2l_useful_flops(p: int) -> int:
    """FP64 operations the M2L kernel must execute per ilist pair (scalar
    charges, potential + field), counted on the nonzero operator entries of
    its formulation: rotation of the order-p multipole (orders n <= p, real
    (n+1)^2 blocks on the re and im parts), z-translation into the field
    local (target orders <= p+1, source orders <= p-1) plus the potential
    local's order-p source column, inverse rotation of both locals (orders
    <= p and <= p+1), the phase factors in and out (complex products) and the
    additions into the targets."""
    T, T1 = (p + 1) * (p + 2) // 2, (p + 2) * (p + 3) // 2
    rot = 2 * sum((n + 1) ** 2 for n in range(p + 1))
    tz = 2 * (sum((p + 2 - k) * (p - k) for k in range(p)) + sum(p + 1 - k for k in range(p + 1)))
    inv = 2 * sum((j + 1) ** 2 for j in range(p + 1)) + 2 * sum((j + 1) ** 2 for j in range(p + 2))
    return 2 * (rot + tz + inv) + 6 * T + 6 * (T + T1) + 2 * (T + T1)


def m2l_mma_flops(p: int) -> int:
    """FP64 tensor-core operations the M2L kernel (k_m2l_mma) issues per
    ilist pair: its compile-time MMA schedule for one 8-column tile (8x8x4
    DMMA, 512 flops each, zero-padded operator fragments) over 8 columns."""
    rt = lambda n: (n + 8) // 8  # noqa: E731
    kc = lambda n: (n + 4) // 4  # noqa: E731
    rot = sum(2 * rt(n) * kc(n) for n in range(p + 1))
    tz = sum(((p + 2 - k + 7) // 8) * 2 * ((p - k + 3) // 4 if k < p else 0) for k in range(p + 2))
    inv = sum(rt(j) * kc(j) * 2 * (1 if j == p + 1 else 2) for j in range(p + 2))
    return (rot + tz + inv) * 512 // 8


def measured_peaks() -> tuple[dict, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return json.loads(f.read_text()), "measured (MEASURED_PEAKS.json)"
        except ValueError:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback (earlier measurement on this pool)"


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


def int8_peak_tops(torch) -> float:
    """Measured int8 dense GEMM rate (cuBLASLt through torch._int_mm, int32
    accumulation), best of 3."""
    n = 8192
    a = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-128, 127, (n, n), dtype=torch.int8, device="cuda")
    torch._int_mm(a, b)
    best = 0.0
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def m2l_i8_ops(p: int) -> int:
    """int8 tensor-core operations of the mixed plans' M2L (k_m2l_i8) per
    ilist pair and charge component, on the nonzero entries of its dense
    operator: potential-local rows (p+1)^2 x (p+1)^2 moments, field-local
    rows (p+2)^2 x p^2, each a product of four-digit numbers taken as ten
    8-bit digit products (2 ops per multiply-add)."""
    return 2 * 10 * ((p + 1) ** 4 + (p + 2) ** 2 * p ** 2)


DATA_DESC = {
    "plummer": "synthetic (seeded Plummer sphere, a=1, r<=10; charges U[-1,1])",
    "uniform": "synthetic (seeded uniform unit cube; charges U[-1,1])",
    "shell": "synthetic (seeded thin spherical shell r=1, thickness 0.01; charges U[-1,1])",
    "gauss2": "synthetic (seeded two Gaussian clusters sigma 0.05, centres 0.5 apart, clipped; charges U[-1,1])",
}


def reference_solve(pos, q, p: int, cores: int, leaf: int = LEAF):
    """One solve of the reference's own CPU implementation (the compiled,
    unmodified reference headers: tree + FMM3D set-up + rinv for the
    potential, FMM3D<3, grad> set-up + two rinv<true> runs for the field),
    as `cores` shim ranks (mpirun -n cores).  Returns (seconds, phases)."""
    from oracle import refio

    out = refio.run_reference(pos, q, p=p, max_level=20, max_ppn=leaf,
                              flags=refio.FLAG_POT | refio.FLAG_FIELD, ranks=cores, timeout=1800)
    ph = {k: out[k] for k in ("T_TREE", "T_CTOR1", "T_POT", "T_CTOR3G", "T_FIELD")}
    return sum(ph.values()), ph


def cpu_baseline(dist: str, n_total: int, n_sample: int, p: int, steps: int = 1, leaf: int = LEAF):
    """The reference's CPU implementation on a bounded sample of the workload
    (the first n_sample of its n_total seeded points and their charges), one
    shim rank per host core; the oracle's restatement on 1 core if the
    compiled reference is absent."""
    from oracle import refio
    from simplefmm_b200 import workloads as W

    cores = host_cores()
    n_sample = min(n_sample, n_total)
    pos = W.points(dist, n_total, SEED)[:n_sample]
    q = W.charges(n_total, SEED)[:n_sample]
    kind = "reference"
    vals = []
    if refio.have_reference():
        for _ in range(steps):
            t, _ = reference_solve(pos, q, p, cores, leaf)
            vals.append(n_sample / t)
    else:
        from oracle import pyoracle
        kind, cores = "port", 1
        for _ in range(steps):
            t0 = time.perf_counter()
            tr = pyoracle.Tree(pos, 20, leaf)
            tr.potential_field(p, q)
            vals.append(n_sample / (time.perf_counter() - t0))
    return vals, {"unit": "points/s", "cores": cores, "kind": kind,
                  "sample": f"first {n_sample} of the workload's {n_total} {dist} points, p={p}, leaf {leaf}, potential + field "
                            f"(tree + FMM3D set-up + rinv, field via two rinv<true> runs)"}


def roofline_i8(torch, pairs: int, p: int, m2l_ms: float, m2l_bytes: int) -> dict:
    """Roofline of the mixed plans' dominant kernel, the int8-slice M2L on
    the tensor cores, against the measured int8 GEMM rate."""
    ops = pairs * m2l_i8_ops(p)
    achieved = ops / (m2l_ms * 1e-3) / 1e12
    peak = int8_peak_tops(torch)
    rows, k = (p + 1) ** 2 + (p + 2) ** 2, (p + 1) ** 2
    # what the instruction shape allows: N = 128 of the 256 an MMA costs the
    # same for (four int32 accumulators fill tensor memory), rows padded to
    # 128, K to 32
    shape = 0.5 * rows / (128 * -(-rows // 128)) * k / (32 * -(-k // 32))
    return {"bound": "tensor", "pipe": "int8 tensor cores (tcgen05.mma kind::i8, M=128 N=128 K=32)", "kernel": "k_m2l_i8",
            "achieved": achieved, "peak": peak, "unit": "TOPS", "frac": achieved / peak,
            "peak_source": "int8 GEMM (torch._int_mm 8192^3, cuBLASLt) measured in this run; MEASURED_PEAKS.json "
                           "has no int8 figure",
            "work": f"ilist pairs x {m2l_i8_ops(p)} int8 ops per pair (nonzero dense-operator entries x 10 digit "
                    f"products x 2), per launch {ops:.4g}; time = mean CUDA-event M2L phase (moment digits included)",
            "frac_of_shape_bound": achieved / peak / shape, "shape_bound": shape,
            "traffic": None, "traffic_model_bytes": m2l_bytes,
            "traffic_note": "measured DRAM bytes per launch come from an ncu capture (profiles/), not from this run"}


def run_reference_arm(args):
    """The reference's own CPU implementation on this arm's workload: the
    first --ref-sample points (and their charges) of the same seeded point
    set, p and leaf size, potential + field, as one shim rank per host core.
    A full solve of the 4M-point workload did not finish in 20 minutes on the
    16 host cores of a B200 machine (1M points take 24 s there, 75 s on an
    8-core workstation), so each step is this bounded sample; one solve is
    timed per step after the warm-up solves."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import refio
    from simplefmm_b200 import workloads as W

    cores = host_cores()
    if not refio.have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference (oracle/_ref/ref_driver) not built"}),
              flush=True)
        return
    n = min(args.ref_sample or args.n, args.n)
    pos = W.points(args.dist, args.n, SEED)[:n]
    q = W.charges(args.n, SEED)[:n]
    vals, phases = [], []
    for i in range(args.warmup + args.steps):
        t, ph = reference_solve(pos, q, args.p, cores, args.leaf)
        if i >= args.warmup:
            vals.append(n / t)
            phases.append(ph)
    v = statistics.median(vals)
    same = n == args.n
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": DATA_DESC.get(args.dist, args.dist),
            "config": workload_config(args, args.n, 1),
            "same_config": same,
            "sample": (f"the full workload" if same else
                       f"first {n} of the workload's {args.n} points (same seeded set and charges), p={args.p}, "
                       f"leaf {args.leaf}, potential + field; the full solve does not finish within minutes on these cores"),
            "reference_phases_s": phases[-1] if phases else None,
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": cores, "kind": "reference",
                             "sample": f"{n} points, tree + FMM3D set-up + rinv (potential) + FMM3D<3,grad> set-up "
                                       f"+ two rinv<true> (field), {cores} shim ranks"},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def small_solves_bench(args):
    """Costs of small solves (the serving regime), Plummer points, leaf 64,
    p = args.p, potential + field, FP64, host arrays: for each size the
    median over 9 repetitions (after 3) of the wall time of the tree build,
    the plan set-up and the evaluation, and the device time of the build
    (fmm_tree_build_phases summed); then the per-solve wall time of a plain
    solve, a batch of one and a batch of eight copies (fmm_solve_batch)."""
    import simplefmm_b200 as sf
    from simplefmm_b200 import workloads as W

    ctx = sf.Context(0)
    reps, skip = 12, 3
    single = {}
    for n in (2000, 10000, 50000, 400000):
        pos, q = W.points("plummer", n, 3), W.charges(n, 3)
        rows = []
        for _ in range(reps):
            t0 = time.perf_counter()
            tree = sf.Tree(pos, 20, LEAF, ctx=ctx)
            t1 = time.perf_counter()
            plan = sf.Plan(tree, args.p, 1)
            t2 = time.perf_counter()
            plan.evaluate(q, np.zeros(n), np.zeros((n, 3)))
            t3 = time.perf_counter()
            ph = tree.build_phases()
            rows.append(((t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3, sum(v[0] for v in ph.values()), ph))
            plan.close()
            tree.close()
        med = lambda k: round(statistics.median(r[k] for r in rows[skip:]), 4)  # noqa: E731
        single[n] = {"build_wall_ms": med(0), "plan_wall_ms": med(1), "evaluate_wall_ms": med(2),
                     "build_device_ms": med(3),
                     "build_phases_ms": {k: round(statistics.median(r[4][k][0] for r in rows[skip:]), 4)
                                         for k in rows[0][4]}}
    batch = {}
    for n in (2000, 10000, 50000):
        pos, q = W.points("plummer", n, 3), W.charges(n, 3)
        res = {}
        for mode, count in (("plain", 1), ("batch1", 1), ("batch8", 8)):
            ts = []
            for _ in range(15):
                t0 = time.perf_counter()
                if mode == "plain":
                    tree = sf.Tree(pos, 20, LEAF, ctx=ctx)
                    sf.Plan(tree, args.p, 1).evaluate(q, np.zeros(n), np.zeros((n, 3)))
                    tree.close()
                else:
                    sf.solve_batch([(pos, q)] * count, args.p, ctx=ctx)
                ts.append((time.perf_counter() - t0) * 1e3)
            res[mode + "_ms_per_solve"] = round(statistics.median(ts[3:]) / count, 4)
        batch[n] = res
    print(json.dumps({"metric": "small-solve costs (wall ms, host arrays)", "p": args.p, "leaf": LEAF,
                      "distribution": "plummer", "single": single, "per_solve": batch,
                      "batch_graphs": sf.batch_graph_stats(ctx)}), flush=True)


def workload_config(args, n: int, world: int) -> dict:
    par = f"shard x{world} (one solve, NCCL all-reduce)" if getattr(args, "shard", False) and world > 1 else f"replicas x{world}"
    leaf = getattr(args, "leaf", LEAF)
    return {"workload": f"{args.dist}_n{n}_p{args.p}_leaf{leaf}_{args.precision}_potential+field", "n": n,
            "p": args.p, "leaf": leaf, "distribution": args.dist, "precision": args.precision,
            "parallelism": par, "l2": "flushed (256 MiB write) between timed steps"}


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
        st = dict(srv.stats(), **srv.batch_stats())
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
        "dtype": "f64" if args.precision == "fp64" else (
            "f32 near field; M2L in int8 slices on the tensor cores (32-bit fixed point, exact int32 sums); "
            "f64 moments, locals and sums"),
        "data": "synthetic (seeded; Poisson arrivals; N log-uniform [1e3, 1e6]; uniform / Plummer / shell; p in {6, 10})",
        "batching": "requests of <= 65,536 points solved in batches sharing one plan and one graph-launched evaluation",
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
    ap.add_argument("--leaf", type=int, default=LEAF, help="max points per leaf (max_particles_per_node)")
    ap.add_argument("--dist", default="plummer")
    ap.add_argument("--ref-sample", type=int, default=1_000_000,
                    help="reference arm: the first this many points of the workload (0 = all of it)")
    ap.add_argument("--cpu-sample", type=int, default=400_000, help="cpu_baseline leg: points of its bounded sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip timing the mixed-precision form beside the FP64 step")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--serve", action="store_true", help="serving-stream benchmark instead of the solve benchmark")
    ap.add_argument("--small", action="store_true",
                    help="small-solve costs instead of the solve benchmark: tree build, plan set-up and evaluation "
                         "of single solves, and the per-solve time of batches (fmm_solve_batch)")
    ap.add_argument("--shard", action="store_true",
                    help="with --gpus N > 1: one solve split over the N ranks (fmm_plan_set_shard, NCCL all-reduce of "
                         "moments, locals and outputs; strong scaling) instead of N independent replicas")
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
    if args.small:
        small_solves_bench(args)
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
    sharded = args.shard and world > 1

    def step(precision=None):
        # one evaluation as a time-stepping caller runs it: release the
        # previous step's tree and plan, build the tree, set up, evaluate
        while live:
            live.pop().close()
        pot_d.zero_()
        fld_d.zero_()
        tree = sf.Tree(pos_d, 20, args.leaf, ctx=ctx)
        plan = sf.Plan(tree, p, 1, precision=precision or args.precision)
        if sharded:
            plan.set_shard(rank, world)
            plan.evaluate_sharded(q_d, pot_d, fld_d, allreduce=dist.all_reduce)
            dist.all_reduce(pot_d)
            dist.all_reduce(fld_d)
        else:
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
    value = n * (1 if sharded else world) * args.steps / (total_ms * 1e-3)

    # accuracy of the last step against the FP64 direct sum on seeded targets
    n_check = min(n, 10_000)
    tg = np.random.default_rng(SEED).choice(n, n_check, replace=False)
    dpot, dfld = sf.direct(pos_h, q_h, tg, ctx=ctx)
    pot_h, fld_h = pot_d.cpu().numpy(), fld_d.cpu().numpy()
    err_pot = float(np.linalg.norm(pot_h[tg] - dpot) / np.linalg.norm(dpot))
    err_fld = float(np.linalg.norm(fld_h[tg] - dfld) / np.linalg.norm(dfld))

    stats = tree.stats()
    depth = tree.depth
    m2l_avg = statistics.mean(m2l_ms)
    pairs = stats["ilist_pairs"]
    useful = pairs * m2l_useful_flops(p)                # per launch
    achieved = useful / (m2l_avg * 1e-3) / 1e12
    peak = fp64_peak_tflops(torch)
    tensor_i8 = args.precision == "mixed" and 2 <= p <= 12
    peaks, peaks_src = measured_peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    T, T1 = (p + 1) * (p + 2) // 2, (p + 2) * (p + 3) // 2
    # M2L bytes that must cross HBM at least once per launch: every node's
    # moments read, both locals of every node written, the ilist entries read
    m2l_bytes = stats["nodes"] * 16 * (T + T + T1) + 8 * pairs
    build = {}
    for name, (ms, by) in tree.build_phases().items():
        gbs = by / (ms * 1e-3) / 1e9 if ms > 0 else None
        build[name] = {"ms": round(ms, 4), "bytes": int(by), "gbs": gbs, "frac_hbm": gbs / hbm if gbs else None}

    e2e = None
    if not args.no_e2e:
        # the same step through the public API with pinned host arrays: the
        # host->device copies of the inputs (and of the accumulated outputs)
        # and the device->host copy of the outputs are inside the timed region
        pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
        pos_p, q_p = pin(pos_h), pin(q_h)
        pot_p, fld_p = pin(np.zeros(n)), pin(np.zeros((n, 3)))
        ctx2 = sf.Context(local)
        if sharded:
            ctx2.set_stream(stream.cuda_stream)

        def e2e_step():
            if not sharded:
                tr = sf.Tree(pos_p, 20, args.leaf, ctx=ctx2)
                sf.Plan(tr, p, 1, precision=args.precision).evaluate(q_p, pot_p, fld_p)
                return tr
            pos_x = torch.from_numpy(pos_p).cuda(non_blocking=True)
            q_x = torch.from_numpy(q_p).cuda(non_blocking=True)
            pot_x = torch.from_numpy(pot_p).cuda(non_blocking=True)
            fld_x = torch.from_numpy(fld_p).cuda(non_blocking=True)
            tr = sf.Tree(pos_x, 20, args.leaf, ctx=ctx2)
            pl = sf.Plan(tr, p, 1, precision=args.precision).set_shard(rank, world)
            pot_0, fld_0 = pot_x.clone(), fld_x.clone()
            pl.evaluate_sharded(q_x, pot_x, fld_x, allreduce=dist.all_reduce)
            pot_x.sub_(pot_0)                          # this shard's increments, summed over the shards
            fld_x.sub_(fld_0)
            dist.all_reduce(pot_x)
            dist.all_reduce(fld_x)
            pot_p[:] += pot_x.cpu().numpy()
            fld_p[:] += fld_x.cpu().numpy()
            return tr

        e2e_step().close()
        et = []
        for _ in range(args.steps):
            pot_p[:] = 0
            fld_p[:] = 0
            flush.zero_()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            tr = e2e_step()
            torch.cuda.synchronize()
            et.append(time.perf_counter() - t0)
            tr.close()
        e2e_s = statistics.mean(et)
        if world > 1:
            tt = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_s = float(tt.item())
        e2e = {"value": n * (1 if sharded else world) / e2e_s, "unit": "points/s",
               "h2d_bytes_per_step": int(pos_p.nbytes + q_p.nbytes + pot_p.nbytes + fld_p.nbytes),
               "d2h_bytes_per_step": int(pot_p.nbytes + fld_p.nbytes)}

    # the mixed-precision form on the same workload, in the same run: the same
    # step (tree, plan, evaluation), timed the same way, checked against the
    # same direct-sum targets
    mixed = None
    if args.precision == "fp64" and world == 1 and not args.no_mixed:
        for _ in range(args.warmup):
            step("mixed")
            flush.zero_()
        torch.cuda.synchronize()
        mt = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            _, mplan = step("mixed")
            e_.record(stream)
            e_.synchronize()
            mt.append(s_.elapsed_time(e_))
        mtm = mplan.timings()
        mpot, mfld = pot_d.cpu().numpy(), fld_d.cpu().numpy()
        m_ms = sum(mt) / len(mt)
        mixed = {"value": n / (m_ms * 1e-3), "unit": "points/s", "ms_per_step": m_ms,
                 "speedup_vs_fp64": (total_ms / args.steps) / m_ms,
                 "rel_error_vs_direct": {"potential": float(np.linalg.norm(mpot[tg] - dpot) / np.linalg.norm(dpot)),
                                         "field": float(np.linalg.norm(mfld[tg] - dfld) / np.linalg.norm(dfld)),
                                         "targets": n_check},
                 "rel_l2_vs_fp64_path": {"potential": float(np.linalg.norm(mpot - pot_h) / np.linalg.norm(pot_h)),
                                         "field": float(np.linalg.norm(mfld - fld_h) / np.linalg.norm(fld_h))},
                 "m2l_ms": mtm["m2l_ms"], "p2p_ms": mtm["p2p_ms"],
                 "dtype": "f32 near field; M2L in int8 slices on the tensor cores (32-bit fixed point, exact int32 sums); "
                          "f64 moments, locals and sums"}
        while live:
            live.pop().close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        vals, info = cpu_baseline(args.dist, n, args.cpu_sample, p, leaf=args.leaf)
        cpu = dict(info, value=statistics.median(vals))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else (
                "f32 near field; M2L in int8 slices on the tensor cores (32-bit fixed point, exact int32 sums); "
                "f64 moments, locals and sums"),
            "data": DATA_DESC.get(args.dist, f"synthetic (seeded {args.dist})"),
            "config": workload_config(args, n, world),
            "tree": {"depth": depth, **stats},
            "rel_error_vs_direct": {"potential": err_pot, "field": err_fld, "targets": n_check},
            "phases_ms": {k: round(statistics.mean(ph[k] for ph in phases), 3) for k in phases[0]},
            "step_ms": [round(x, 3) for x in times],
            "tree_ms_per_step": [round(ph["tree_ms"], 3) for ph in phases],
            "tree_build_phases": dict(build, peak_hbm_gbs=hbm, peak_source=peaks_src,
                                      work="algorithmic bytes of each phase (fmm_tree_build_phases) / its device time"),
            "roofline": roofline_i8(torch, pairs, p, m2l_avg, m2l_bytes) if tensor_i8 else {
                         "bound": "tensor", "pipe": "FP64 tensor cores (DMMA 8x8x4)", "kernel": "k_m2l_mma",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "FP64 DGEMM (torch float64 matmul 8192^3, cuBLAS DMMA) measured in this run; "
                                        "MEASURED_PEAKS.json has no FP64 figure",
                         "work": f"ilist pairs x {m2l_useful_flops(p)} useful FP64 flops per pair (nonzero operator "
                                 f"entries of rotate / translate / rotate back, phases, sums), per launch "
                                 f"{useful:.4g} flops; time = mean CUDA-event M2L phase",
                         "frac_mma": pairs * m2l_mma_flops(p) / (m2l_avg * 1e-3) / 1e12 / peak,
                         "mma_flops_per_pair": m2l_mma_flops(p),
                         "frac_ref_ops": pairs * 4 * f_m2l(p) / (m2l_avg * 1e-3) / 1e12 / peak,
                         "ref_ops_per_pair": 4 * f_m2l(p),
                         "traffic": None,
                         "traffic_model_bytes": m2l_bytes,
                         "traffic_note": "measured DRAM bytes per launch come from an ncu capture (profiles/), "
                                         "not from this run"},
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": int(launches),
            "mixed": mixed,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
