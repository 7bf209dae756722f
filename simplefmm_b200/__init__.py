"""simplefmm_b200 -- B200-native 3D Laplace FMM behind a C ABI.

Two layers over ``libsimplefmm_b200.so`` (include/simplefmm_b200.h):

* ``Context`` / ``Tree`` / ``Plan`` -- thin handles on the C ABI;
* ``Box`` / ``OctreePartitioner`` / ``FMM3D`` -- the reference library's own
  API (box.hpp:84, partition.hpp:397-446, fmm.hpp:204-881) with the same
  names, argument meaning and accumulate-into-U semantics, so code written
  against the reference reads the same.

There is no CPU fallback: without the compiled library or a CUDA device the
calls raise ``FMMError``.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

__all__ = ["FMMError", "Context", "Tree", "Plan", "Box", "OctreePartitioner", "OctreeLevel", "FMM3D",
           "direct", "launch_count", "load_library", "LIB_PATH", "Server"]

LIB_PATH = Path(__file__).resolve().parent / "libsimplefmm_b200.so"

HOST, DEVICE = 0, 1
PRECISION = {"fp64": 0, "mixed": 1}

EXPORT = dict(node_keys=0, leaf_nodes=1, index_ptr=2, index=3, ilist_ptr=4, ilist=5, clist_ptr=6, clist=7,
              plist=8, nlist_ptr=9, nlist=10, partitions=11)
_EXPORT_DTYPE = {0: np.int64, 7: np.int64, 8: np.int64}

_lib = None


class FMMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def load_library():
    """Load the compiled library (fails loudly when it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FMMError(-1, f"{LIB_PATH} is not built (python -m simplefmm_b200.build)")
    L = C.CDLL(str(LIB_PATH))
    vp, i64, dbl, i32 = C.c_void_p, C.c_int64, C.c_double, C.c_int
    sig = {
        "fmm_status_string": ([i32], C.c_char_p),
        "fmm_last_error": ([], C.c_char_p),
        "fmm_version": ([], C.c_char_p),
        "fmm_context_create": ([i32, C.POINTER(vp)], i32),
        "fmm_context_destroy": ([vp], i32),
        "fmm_context_set_stream": ([vp, vp], i32),
        "fmm_context_synchronize": ([vp], i32),
        "fmm_host_register": ([vp, C.c_size_t], i32),
        "fmm_host_unregister": ([vp], i32),
        "fmm_tree_build": ([vp, vp, i64, i32, i32, i32, i32, dbl, C.POINTER(vp)], i32),
        "fmm_tree_destroy": ([vp], i32),
        "fmm_tree_build_box": ([vp, vp, i64, i32, C.POINTER(dbl), dbl, i32, i32, i32, dbl, C.POINTER(vp)], i32),
        "fmm_plan_set_exclusions": ([vp, vp, vp, i32, i32], i32),
        "fmm_plan_set_m2l": ([vp, i32], i32),
        "fmm_plan_set_shard": ([vp, i32, i32], i32),
        "fmm_evaluate_stage": ([vp, vp, vp, vp, i32], i32),
        "fmm_plan_exchange_buffer": ([vp, i32, C.POINTER(vp), C.POINTER(i64)], i32),
        "fmm_plan_capture": ([vp, vp, vp, vp], i32),
        "fmm_plan_replay": ([vp], i32),
        "fmm_tree_depth": ([vp, C.POINTER(i32)], i32),
        "fmm_tree_box": ([vp, C.POINTER(dbl), C.POINTER(dbl)], i32),
        "fmm_tree_export_size": ([vp, i32, i32, C.POINTER(i64)], i32),
        "fmm_tree_export": ([vp, i32, i32, vp], i32),
        "fmm_tree_stats": ([vp, C.POINTER(i64)], i32),
        "fmm_tree_build_phases": ([vp, C.POINTER(dbl), C.POINTER(dbl)], i32),
        "fmm_plan_create": ([vp, i32, i32, i32, C.POINTER(vp)], i32),
        "fmm_plan_destroy": ([vp], i32),
        "fmm_rinv": ([vp, vp, vp, i32, i32], i32),
        "fmm_evaluate": ([vp, vp, vp, vp, i32], i32),
        "fmm_plan_timings": ([vp, C.POINTER(dbl)], i32),
        "fmm_direct": ([vp, vp, i64, vp, i32, vp, i64, vp, vp, i32], i32),
        "fmm_direct_noalloc": ([vp, i64, vp, i32, vp, i64, vp, vp, vp], i32),
        "fmm_launch_count": ([C.POINTER(i64)], i32),
        "fmm_server_create": ([i32, i32, C.c_size_t, C.POINTER(vp)], i32),
        "fmm_server_destroy": ([vp], i32),
        "fmm_server_submit": ([vp, vp, i64, vp, i32, i32, i32, i32, vp, vp, C.POINTER(i64)], i32),
        "fmm_server_poll": ([vp, i64, C.POINTER(i32)], i32),
        "fmm_server_wait": ([vp, i64, C.POINTER(dbl)], i32),
        "fmm_server_stats": ([vp, C.POINTER(dbl)], i32),
        "fmm_server_memory": ([vp, C.POINTER(dbl)], i32),
        "fmm_solve_batch": ([vp, vp, i32, i32, i32, i32, i32], i32),
        "fmm_server_batch_stats": ([vp, C.POINTER(i64), C.POINTER(i64)], i32),
        "fmm_batch_graph_stats": ([vp, C.POINTER(i64), C.POINTER(i64)], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


class _DeviceArray:
    """A float64 device array by address, for torch.as_tensor."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                         "strides": None}


def _check(rc: int):
    if rc != 0:
        L = load_library()
        raise FMMError(rc, f"{L.fmm_status_string(rc).decode()}: {L.fmm_last_error().decode()}")


def _ptr(a):
    """(address, where) of a numpy array (host) or CUDA tensor / __cuda_array_interface__ (device)."""
    if a is None:
        return None, HOST
    if isinstance(a, np.ndarray):
        return a.ctypes.data, HOST
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        return cai["data"][0], DEVICE
    if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False):
        return a.data_ptr(), DEVICE
    raise TypeError("expected a numpy array or a CUDA tensor")


class Context:
    """One device + one stream; trees and plans built on it share both."""

    def __init__(self, device: int = 0):
        L = load_library()
        h = C.c_void_p()
        _check(L.fmm_context_create(device, C.byref(h)))
        self._h = h
        self.device = device

    def set_stream(self, stream_handle: int):
        _check(load_library().fmm_context_set_stream(self._h, C.c_void_p(stream_handle)))

    def synchronize(self):
        _check(load_library().fmm_context_synchronize(self._h))

    def close(self):
        if getattr(self, "_h", None):
            load_library().fmm_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class Tree:
    """Box + adaptive octree + lists, built and kept on the device."""

    def __init__(self, positions, max_level: int = 20, max_particles_per_node: int = 64, vertical_axis: int = 2,
                 phideg: float = 0.0, ctx: Context | None = None, box=None):
        """box = (corner[3], width) gives the root cube explicitly (Box(corner, width, ...));
        otherwise it is fitted to the points."""
        self.ctx = ctx or default_context()
        if isinstance(positions, np.ndarray):
            positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        n = int(positions.shape[0])
        addr, where = _ptr(positions)
        h = C.c_void_p()
        L = load_library()
        if box is None:
            _check(L.fmm_tree_build(self.ctx._h, C.c_void_p(addr), n, where, max_level,
                                    max_particles_per_node, vertical_axis, float(phideg), C.byref(h)))
        else:
            corner = (C.c_double * 3)(*[float(x) for x in box[0]])
            _check(L.fmm_tree_build_box(self.ctx._h, C.c_void_p(addr), n, where, corner, float(box[1]), max_level,
                                        max_particles_per_node, vertical_axis, float(phideg), C.byref(h)))
        self._h = h
        self.n = n
        self.max_level, self.max_ppn = max_level, max_particles_per_node
        self.vertical_axis, self.phideg = vertical_axis, phideg

    @property
    def depth(self) -> int:
        d = C.c_int()
        _check(load_library().fmm_tree_depth(self._h, C.byref(d)))
        return d.value

    def box(self):
        w = C.c_double()
        c = (C.c_double * 3)()
        _check(load_library().fmm_tree_box(self._h, C.byref(w), c))
        return w.value, np.array(list(c))

    def stats(self) -> dict:
        s = (C.c_int64 * 5)()
        _check(load_library().fmm_tree_stats(self._h, s))
        return dict(nodes=s[0], leaves=s[1], ilist_pairs=s[2], near_pairs=s[3], near_ranges=s[4])

    PHASES = ("keys", "refine", "leaves_points", "colleagues", "ilist", "near_lists")

    def build_phases(self) -> dict:
        """Device ms and algorithmic bytes of each tree-build phase:
        {phase: (ms, bytes)} (fmm_tree_build_phases)."""
        ms, by = (C.c_double * 6)(), (C.c_double * 6)()
        _check(load_library().fmm_tree_build_phases(self._h, ms, by))
        return {k: (ms[i], by[i]) for i, k in enumerate(self.PHASES)}

    def export(self, level: int, what) -> np.ndarray:
        w = EXPORT[what] if isinstance(what, str) else int(what)
        cnt = C.c_int64()
        _check(load_library().fmm_tree_export_size(self._h, level, w, C.byref(cnt)))
        if cnt.value < 0:
            raise FMMError(1, f"export {what} is not defined at level {level}")
        out = np.zeros(max(cnt.value, 1), dtype=_EXPORT_DTYPE.get(w, np.int32))
        if cnt.value > 0:
            _check(load_library().fmm_tree_export(self._h, level, w, C.c_void_p(out.ctypes.data)))
        return out[:cnt.value]

    def dump(self) -> dict:
        """Tree in the reference driver's dump format (keys CNODE<l>, ILEAF<l>, ...)."""
        w, c = self.box()
        D = self.depth
        d = {"BOX": np.array([w, *c]), "DEPTH": np.array([D, 1], np.int32)}
        for l in range(D + 1):
            d[f"CNODE{l}"] = self.export(l, "node_keys")
            d[f"ILEAF{l}"] = self.export(l, "leaf_nodes")
            d[f"IDXP{l}"] = self.export(l, "index_ptr")
            d[f"IDXV{l}"] = self.export(l, "index")
            if l >= 2:
                d[f"ILP{l}"] = self.export(l, "ilist_ptr")
                d[f"ILV{l}"] = self.export(l, "ilist")
            if l < D:
                d[f"CLP{l}"] = self.export(l, "clist_ptr")
                d[f"CLV{l}"] = self.export(l, "clist")
            if l >= 1:
                d[f"PL{l}"] = self.export(l, "plist")
            d[f"NLP{l}"] = self.export(l, "nlist_ptr")
            d[f"NLV{l}"] = self.export(l, "nlist")
        d["PARTS"] = self.export(0, "partitions")
        return d

    def close(self):
        if getattr(self, "_h", None):
            load_library().fmm_tree_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """Operators of order p for one tree (the FMM3D object)."""

    def __init__(self, tree: Tree, p: int, qdim: int = 1, precision: str = "fp64"):
        self.tree = tree
        self.p, self.qdim = p, qdim
        h = C.c_void_p()
        _check(load_library().fmm_plan_create(tree._h, p, qdim, PRECISION[precision], C.byref(h)))
        self._h = h

    def set_shard(self, index: int, count: int):
        """This plan's share of one solve split over `count` devices
        (fmm_plan_set_shard); evaluate it with evaluate_sharded."""
        _check(load_library().fmm_plan_set_shard(self._h, index, count))
        return self

    def exchange_buffer(self, which: int):
        """Device buffer `which` (0 moments, 1 potential locals, 2 field
        locals) as a flat float64 CUDA tensor sharing the plan's memory."""
        import torch

        ptr, cnt = C.c_void_p(), C.c_int64()
        _check(load_library().fmm_plan_exchange_buffer(self._h, which, C.byref(ptr), C.byref(cnt)))
        return torch.as_tensor(_DeviceArray(ptr.value, cnt.value), device="cuda")

    def evaluate_stage(self, Q, pot, field, stage: int):
        """One stage (0, 1, 2) of a sharded evaluation on CUDA tensors."""
        ptrs = []
        for arr in (Q, pot, field):
            addr, where = _ptr(arr)
            if arr is not None and where != DEVICE:
                raise FMMError(1, "sharded evaluation takes device arrays")
            ptrs.append(C.c_void_p(addr) if arr is not None else None)
        _check(load_library().fmm_evaluate_stage(self._h, *ptrs, stage))

    def evaluate_sharded(self, Q, pot=None, field=None, allreduce=None):
        """All three stages of this shard's share; allreduce(tensor) must sum
        a tensor in place over the shards (e.g. torch.distributed.all_reduce
        on NCCL) -- it runs on the moments after stage 0 and on both locals
        after stage 1.  pot / field receive this shard's points' results."""
        self.evaluate_stage(Q, pot, field, 0)
        allreduce(self.exchange_buffer(0))
        self.evaluate_stage(Q, pot, field, 1)
        allreduce(self.exchange_buffer(1))
        allreduce(self.exchange_buffer(2))
        self.evaluate_stage(Q, pot, field, 2)

    def set_m2l(self, method: str):
        """M2L formulation: "rotation" (default) or "direct", the reference's
        FMM_M2L_DIRECT option (fmm_plan_set_m2l)."""
        _check(load_library().fmm_plan_set_m2l(self._h, {"rotation": 0, "direct": 1}[method]))
        return self

    def evaluate(self, Q, pot=None, field=None):
        """pot += potential, field += field (either may be None).  numpy arrays
        run synchronously through host staging; CUDA tensors run on the
        context's stream."""
        qa, wq = _ptr(Q)
        pa, wp = _ptr(pot)
        fa, wf = _ptr(field)
        where = wq
        for a, w in ((pa, wp), (fa, wf)):
            if a is not None and w != where:
                raise TypeError("Q and outputs must all be host arrays or all device arrays")
        if where == HOST:
            Q = np.ascontiguousarray(Q, dtype=np.float64)
            qa = Q.ctypes.data
            for arr in (pot, field):
                if arr is not None and not (arr.flags.c_contiguous and arr.dtype == np.float64):
                    raise TypeError("outputs must be C-contiguous float64 arrays")
        _check(load_library().fmm_evaluate(self._h, C.c_void_p(qa), C.c_void_p(pa) if pa else None,
                                           C.c_void_p(fa) if fa else None, where))

    def rinv(self, Q, U, gradient: bool = False):
        """FMM3D::rinv (gradient False) / rinv<true> (fmm.hpp:864-881): U += ..."""
        qa, wq = _ptr(Q)
        ua, wu = _ptr(U)
        if wq != wu:
            raise TypeError("Q and U must both be host arrays or both device arrays")
        if wq == HOST:
            Q = np.ascontiguousarray(Q, dtype=np.float64)
            qa = Q.ctypes.data
        _check(load_library().fmm_rinv(self._h, C.c_void_p(qa), C.c_void_p(ua), int(bool(gradient)), wq))

    def set_exclusions(self, row_ptr, cols, near_too: bool = True):
        """Excluded sources per target (CSR over original indices); None clears.
        near_too=False: the reference's slist under the default is_self."""
        L = load_library()
        if row_ptr is None:
            _check(L.fmm_plan_set_exclusions(self._h, None, None, HOST, 0))
            return
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        cl = np.ascontiguousarray(cols, dtype=np.int32)
        _check(L.fmm_plan_set_exclusions(self._h, C.c_void_p(rp.ctypes.data), C.c_void_p(cl.ctypes.data), HOST,
                                         int(bool(near_too))))

    def capture(self, Q, pot=None, field=None):
        """Capture evaluate(Q, pot, field) on device arrays as a CUDA graph (see replay)."""
        ptrs = []
        for arr in (Q, pot, field):
            addr, where = _ptr(arr)
            if arr is not None and where != DEVICE:
                raise FMMError(1, "capture takes device arrays")
            ptrs.append(C.c_void_p(addr) if arr is not None else None)
        _check(load_library().fmm_plan_capture(self._h, *ptrs))

    def replay(self):
        """Launch the captured evaluation again (asynchronous on the context's stream)."""
        _check(load_library().fmm_plan_replay(self._h))

    def timings(self) -> dict:
        t = (C.c_double * 6)()
        _check(load_library().fmm_plan_timings(self._h, t))
        return dict(upward_ms=t[0], m2l_ms=t[1], downward_ms=t[2], p2p_ms=t[3], evaluate_ms=t[4], tree_ms=t[5])

    def close(self):
        if getattr(self, "_h", None):
            load_library().fmm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def direct(positions, Q, targets, pot=True, field=True, ctx: Context | None = None):
    """FP64 direct sums at ``targets`` on the device (main.cpp:70-111).
    Returns (pot, field); numpy in, numpy out."""
    ctx = ctx or default_context()
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    Q = np.ascontiguousarray(Q, dtype=np.float64)
    qdim = 1 if Q.ndim == 1 else Q.shape[1]
    t = np.ascontiguousarray(targets, dtype=np.int64)
    po = np.zeros((t.size, qdim)) if pot else None
    fo = np.zeros((t.size, 3)) if field else None
    _check(load_library().fmm_direct(ctx._h, C.c_void_p(pos.ctypes.data), pos.shape[0], C.c_void_p(Q.ctypes.data),
                                     qdim, C.c_void_p(t.ctypes.data), t.size,
                                     C.c_void_p(po.ctypes.data) if pot else None,
                                     C.c_void_p(fo.ctypes.data) if field else None, HOST))
    if po is not None and qdim == 1:
        po = po[:, 0]
    return po, fo


class _BatchItem(C.Structure):
    _fields_ = [("xyz", C.c_void_p), ("n", C.c_int64), ("Q", C.c_void_p), ("leaf", C.c_int), ("pot", C.c_void_p),
                ("field", C.c_void_p)]


def solve_batch(sets, p: int, qdim: int = 1, precision: str = "fp64", leaf=64, pot=True, field=True,
                ctx: Context | None = None, max_level: int = 20):
    """Solve several independent point sets with one plan (fmm_solve_batch):
    ``sets`` is a list of (positions, charges); ``leaf`` one leaf size or one
    per set.  Returns a list of (pot, field) per set; numpy in, numpy out."""
    ctx = ctx or default_context()
    leaves = list(leaf) if np.ndim(leaf) else [leaf] * len(sets)
    keep, items, outs = [], (_BatchItem * len(sets))(), []
    for k, (pos, Q) in enumerate(sets):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        n = pos.shape[0]
        po = np.zeros((n,) if qdim == 1 else (n, qdim)) if pot else None
        fo = np.zeros((n, 3)) if field else None
        keep += [pos, Q]
        items[k] = _BatchItem(pos.ctypes.data, n, Q.ctypes.data, int(leaves[k]), po.ctypes.data if pot else None,
                              fo.ctypes.data if field else None)
        outs.append((po, fo))
    _check(load_library().fmm_solve_batch(ctx._h, C.cast(items, C.c_void_p), len(sets), p, qdim, PRECISION[precision],
                                          max_level))
    return outs


def batch_graph_stats(ctx: Context | None = None) -> dict:
    """Graph executables the context's batches instantiated and updated in place."""
    ctx = ctx or default_context()
    a, b = C.c_int64(), C.c_int64()
    _check(load_library().fmm_batch_graph_stats(ctx._h, C.byref(a), C.byref(b)))
    return {"instantiated": a.value, "updated": b.value}


class Server:
    """Serving loop (fmm_server_*): submit solves as they arrive; they run
    concurrently on one device under a device-memory budget.  Arrays passed to
    submit() are kept alive until wait()."""

    def __init__(self, device: int = 0, slots: int = 4, memory_budget: int = 16 << 30):
        h = C.c_void_p()
        _check(load_library().fmm_server_create(device, slots, memory_budget, C.byref(h)))
        self._h = h
        self._keep = {}

    def submit(self, positions, Q, p: int, precision: str = "fp64", leaf: int = 0, pot=True, field=True):
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        n = pos.shape[0]
        qdim = 1 if Q.ndim == 1 else Q.shape[1]
        po = np.zeros((n,) if qdim == 1 else (n, qdim)) if pot else None
        fo = np.zeros((n, 3)) if field else None
        rid = C.c_int64()
        _check(load_library().fmm_server_submit(
            self._h, C.c_void_p(pos.ctypes.data), n, C.c_void_p(Q.ctypes.data), qdim, p, PRECISION[precision], leaf,
            C.c_void_p(po.ctypes.data) if pot else None, C.c_void_p(fo.ctypes.data) if field else None, C.byref(rid)))
        self._keep[rid.value] = (pos, Q, po, fo)
        return rid.value

    def done(self, rid: int) -> bool:
        d = C.c_int()
        _check(load_library().fmm_server_poll(self._h, rid, C.byref(d)))
        return bool(d.value)

    def wait(self, rid: int):
        """(pot, field, latency_ms) of request rid."""
        lat = C.c_double()
        try:
            _check(load_library().fmm_server_wait(self._h, rid, C.byref(lat)))
        finally:
            keep = self._keep.pop(rid, None)
        return keep[2], keep[3], lat.value

    def stats(self) -> dict:
        s = (C.c_double * 8)()
        _check(load_library().fmm_server_stats(self._h, s))
        return dict(completed=int(s[0]), p50_ms=s[1], p99_ms=s[2], mean_ms=s[3], peak_running=int(s[4]),
                    peak_bytes=int(s[5]), budget_bytes=int(s[6]), queued=int(s[7]))

    def batch_stats(self) -> dict:
        """Batches of small requests solved together so far (fmm_server_batch_stats)."""
        a, b = C.c_int64(), C.c_int64()
        _check(load_library().fmm_server_batch_stats(self._h, C.byref(a), C.byref(b)))
        return {"batches": a.value, "batched_requests": b.value}

    def memory(self) -> dict:
        """Measured device memory of the running requests (fmm_server_memory)."""
        s = (C.c_double * 3)()
        _check(load_library().fmm_server_memory(self._h, s))
        return dict(peak_measured_bytes=int(s[0]), budget_bytes=int(s[1]), worst_measured_over_estimate=s[2])

    def close(self):
        if getattr(self, "_h", None):
            load_library().fmm_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count() -> int:
    c = C.c_int64()
    _check(load_library().fmm_launch_count(C.byref(c)))
    return c.value


# ---------------------------------------------------------------- reference API
class Box:
    """box.hpp:84-107 -- the root cube of ``positions``.  It is evaluated on the
    device by the partitioner (same arithmetic); ``width()``/``corner()`` are
    available once ``OctreePartitioner.refine`` has run."""

    def __init__(self, positions, vertical_axis: int = 2, phideg: float = 0.0):
        self.positions = positions
        self.vertical_axis, self.phideg = vertical_axis, phideg
        self._tree = None

    def width(self) -> float:
        if self._tree is None:
            raise FMMError(1, "the box is computed by OctreePartitioner.refine")
        return self._tree.box()[0]

    def corner(self) -> np.ndarray:
        if self._tree is None:
            raise FMMError(1, "the box is computed by OctreePartitioner.refine")
        return self._tree.box()[1]


class OctreeLevel:
    """Per-level view (partition.hpp:147-377) exported from the device tree."""

    def __init__(self, tree: Tree, level: int):
        self._t, self._l = tree, level

    def level(self):
        return self._l

    def c_node(self):
        return self._t.export(self._l, "node_keys")

    def n_node(self):
        return int(self.c_node().size)

    def n_leaf(self):
        return int(self._t.export(self._l, "leaf_nodes").size)

    def indices(self):
        return self._t.export(self._l, "index_ptr"), self._t.export(self._l, "index")

    def ilist(self):
        return self._t.export(self._l, "ilist_ptr"), self._t.export(self._l, "ilist").reshape(-1, 4)

    def clist(self):
        return self._t.export(self._l, "clist_ptr"), self._t.export(self._l, "clist").reshape(-1, 2)

    def plist(self):
        return self._t.export(self._l, "plist").reshape(-1, 2)

    def nlist(self):
        return self._t.export(self._l, "nlist_ptr"), self._t.export(self._l, "nlist").reshape(-1, 2)


class OctreePartitioner:
    """partition.hpp:380-500."""

    def __init__(self, positions, box: Box, ctx: Context | None = None):
        self._pos, self._box, self._ctx = positions, box, ctx
        self.tree = None

    def refine(self, max_level: int = 20, max_particles_per_node: int = 64):
        self.tree = Tree(self._pos, max_level, max_particles_per_node, self._box.vertical_axis, self._box.phideg,
                         ctx=self._ctx)
        self._box._tree = self.tree
        return self

    def level(self) -> int:
        return self.tree.depth

    def octreeLevel(self, l: int) -> OctreeLevel:  # noqa: N802 (reference name)
        return OctreeLevel(self.tree, l)

    def get_partition(self, i: int):
        parts = self.tree.export(0, "partitions").reshape(-1, 2)
        return int(parts[i, 0]), int(parts[i, 1])


class FMM3D:
    """FMM3D<double, N, p, Vector, support_gradient> (fmm.hpp:134-882).

    ``rinv(Q, U)`` accumulates the potential of N-component charges,
    ``rinv(Q, U, gradient=True)`` (N = 3) accumulates sum_j Q_j x R/|R|^3,
    as ``rinv<true>``.  ``evaluate(q, pot, field)`` does both in one pass and
    also takes scalar charges for the Coulomb field sum_j q_j R/|R|^3."""

    def __init__(self, partitioner: OctreePartitioner, p: int, N: int = 1, support_gradient: bool = False,
                 comm=None, precision: str = "fp64"):
        if support_gradient and N != 3:
            raise FMMError(2, "support_gradient needs N = 3 (fmm.hpp:550)")
        self.plan = Plan(partitioner.tree, p, N, precision)
        self.p, self.N = p, N

    def rinv(self, Q, U, gradient: bool = False):
        self.plan.rinv(Q, U, gradient)

    def evaluate(self, Q, pot=None, field=None):
        self.plan.evaluate(Q, pot, field)
