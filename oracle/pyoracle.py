"""ctypes wrapper of the CPU restatement (``liboracle.so``) -- TEST ORACLE ONLY.

Returns tree dumps keyed like the reference driver's output (``CNODE<l>``,
``ILEAF<l>``, ``IDXP<l>``/``IDXV<l>``, ``ILP<l>``/``ILV<l>``, ``CLP<l>``/``CLV<l>``,
``PL<l>``, ``NLP<l>``/``NLV<l>``, ``PARTS``, ``BOX``) so tests can compare the
restatement, the compiled reference and the CUDA library field by field.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "liboracle.so"

_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        dp, i64, vp = C.POINTER(C.c_double), C.c_int64, C.c_void_p
        L.oracle_cube.argtypes = [dp, i64, C.c_int, C.c_double, dp]
        L.oracle_key.argtypes = [dp, i64, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int64)]
        L.oracle_key.restype = i64
        L.oracle_tree_build.argtypes = [dp, i64, C.c_int, C.c_int, C.c_int, C.c_double]
        L.oracle_tree_build.restype = vp
        L.oracle_tree_build_box.argtypes = [dp, i64, C.c_int, C.c_int, C.c_int, C.c_double, dp]
        L.oracle_tree_build_box.restype = vp
        L.oracle_tree_free.argtypes = [vp]
        L.oracle_tree_depth.argtypes = [vp]
        L.oracle_tree_export.argtypes = [vp, C.c_int, C.c_int, vp]
        L.oracle_tree_export.restype = i64
        L.oracle_rinv.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp, dp]
        L.oracle_direct.argtypes = [dp, i64, C.c_int, C.c_int, dp, C.POINTER(C.c_int64), i64, dp]
        L.oracle_eval_create.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.oracle_eval_create.restype = vp
        L.oracle_eval_free.argtypes = [vp]
        L.oracle_eval_set_shard.argtypes = [vp, C.c_int, C.c_int]
        L.oracle_eval_stage.argtypes = [vp, C.c_int, dp, dp]
        L.oracle_eval_buffer.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int64)]
        L.oracle_eval_buffer.restype = dp
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def cube(pos, vertical_axis=2, phideg=0.0) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.zeros(4)
    lib().oracle_cube(_dp(pos), pos.shape[0], vertical_axis, phideg, _dp(out))
    return out


def keys(pos, level, vertical_axis=2, phideg=0.0) -> np.ndarray:
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.zeros(pos.shape[0], dtype=np.int64)
    lib().oracle_key(_dp(pos), pos.shape[0], vertical_axis, phideg, level,
                     out.ctypes.data_as(C.POINTER(C.c_int64)))
    return out


class Tree:
    """Restated octree; ``dump()`` mirrors the reference driver's tree sections."""

    def __init__(self, pos, max_level=20, max_ppn=64, vertical_axis=2, phideg=0.0, box=None):
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.n = self.pos.shape[0]
        self.vertical_axis, self.phideg = vertical_axis, phideg
        self._box = None if box is None else np.array([box[1], box[0][0], box[0][1], box[0][2]], dtype=np.float64)
        if box is None:
            self._h = lib().oracle_tree_build(_dp(self.pos), self.n, max_level, max_ppn, vertical_axis, phideg)
        else:
            b4 = np.array([box[0][0], box[0][1], box[0][2], box[1]], dtype=np.float64)
            self._h = lib().oracle_tree_build_box(_dp(self.pos), self.n, max_level, max_ppn, vertical_axis, phideg,
                                                  _dp(b4))
        self.depth = lib().oracle_tree_depth(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_tree_free(h)
            self._h = None

    def _export(self, level, what, dtype):
        n = lib().oracle_tree_export(self._h, level, what, None)
        out = np.zeros(max(n, 0), dtype=dtype)
        if n > 0:
            lib().oracle_tree_export(self._h, level, what, out.ctypes.data_as(C.c_void_p))
        return out

    def dump(self) -> dict:
        box = self._box if self._box is not None else cube(self.pos, self.vertical_axis, self.phideg)
        d = {"BOX": box, "DEPTH": np.array([self.depth, 1], np.int32)}
        for l in range(self.depth + 1):
            d[f"CNODE{l}"] = self._export(l, 0, np.int64)
            d[f"ILEAF{l}"] = self._export(l, 1, np.int32)
            d[f"IDXP{l}"] = self._export(l, 2, np.int32)
            d[f"IDXV{l}"] = self._export(l, 3, np.int32)
            if l >= 2:
                d[f"ILP{l}"] = self._export(l, 4, np.int32)
                d[f"ILV{l}"] = self._export(l, 5, np.int32)
            if l < self.depth:
                d[f"CLP{l}"] = self._export(l, 6, np.int32)
                d[f"CLV{l}"] = self._export(l, 7, np.int64)
            if l >= 1:
                d[f"PL{l}"] = self._export(l, 8, np.int64)
            d[f"NLP{l}"] = self._export(l, 9, np.int32)
            d[f"NLV{l}"] = self._export(l, 10, np.int32)
        d["PARTS"] = self._export(0, 11, np.int32)
        return d

    def rinv(self, p, Q, gradient=False, U=None) -> np.ndarray:
        """Restated ``FMM3D::rinv`` / ``rinv<true>`` (U accumulated, like the reference)."""
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        ncomp = 1 if Q.ndim == 1 else Q.shape[1]
        if U is None:
            U = np.zeros_like(Q)
        rc = lib().oracle_rinv(self._h, p, 1 if gradient else 0, ncomp, _dp(Q), _dp(U))
        if rc != 0:
            raise ValueError("oracle_rinv rejected its arguments")
        return U

    def potential_field(self, p, q):
        """Scalar-charge potential and field E = sum q_j R/|R|^3, the field
        assembled from two ``rinv<true>`` runs with Q=(q,0,0) and (0,0,q)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        pot = self.rinv(p, q)
        z = np.zeros((self.n, 3))
        qx = z.copy(); qx[:, 0] = q
        qz = z.copy(); qz[:, 2] = q
        ux = self.rinv(p, qx, gradient=True)
        uz = self.rinv(p, qz, gradient=True)
        E = np.stack([uz[:, 1], -uz[:, 0], -ux[:, 1]], axis=1)
        return pot, E


def direct(pos, Q, targets, mode="potential") -> np.ndarray:
    """FP64 direct sums at ``targets`` (main.cpp:70-96 plus the scalar field):
    mode 'potential' (sum Q_j/|R|), 'biot' (sum Q_j x R/|R|^3) or 'field'
    (scalar q: sum q_j R/|R|^3) or 'scale' ((n, 2): sum |Q_j|/|R| and
    sum |Q_j|/|R|^2, the per-target magnitudes that bound rounding error)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    Q = np.ascontiguousarray(Q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    ncomp = 1 if Q.ndim == 1 else Q.shape[1]
    m = {"potential": 0, "biot": 1, "field": 2, "scale": 3}[mode]
    nout = 3 if m == 2 else 2 if m == 3 else ncomp
    out = np.zeros((t.shape[0], nout))
    lib().oracle_direct(_dp(pos), pos.shape[0], m, ncomp, _dp(Q), t.ctypes.data_as(C.POINTER(C.c_int64)),
                        t.shape[0], _dp(out))
    return out[:, 0] if (nout == 1) else out


def error_scales(pos, Q, targets=None):
    """(potential scale, field scale) per target: sum_j |Q_j|/r_ij and
    sum_j |Q_j|/r_ij^2 over j != i."""
    if targets is None:
        targets = np.arange(np.asarray(pos).shape[0])
    s = direct(pos, Q, targets, mode="scale")
    return s[:, 0], s[:, 1]


def subtract_exclusions(tree: "Tree", pos, Q, row_ptr, cols, near_too, pot=None, field=None):
    """fmm.hpp:398-408, 773-807: remove the listed pairs (j != i) from results
    computed with the default is_self -- all of them (near_too), or only those
    outside i's near field (the reference's slist).  In place."""
    d = tree.dump()
    parts = d["PARTS"].reshape(-1, 2)
    pos = np.asarray(pos, dtype=np.float64)
    Q = np.asarray(Q, dtype=np.float64)
    n = pos.shape[0]
    for i in range(n):
        li, fi = parts[i]
        ptr, val = d[f"NLP{li}"], d[f"NLV{li}"].reshape(-1, 2)
        near_set = {tuple(x) for x in val[ptr[fi]:ptr[fi + 1]]}
        for e in range(row_ptr[i], row_ptr[i + 1]):
            j = int(cols[e])
            if j == i:
                continue
            if not near_too and tuple(parts[j]) in near_set:
                continue
            R = pos[i] - pos[j]
            r = np.sqrt(R @ R)
            if pot is not None:
                pot[i] -= Q[j] / r
            if field is not None:
                if Q.ndim == 1:
                    field[i] -= Q[j] * R / r**3
                else:
                    field[i] -= np.cross(Q[j], R) / r**3


class ShardedEval:
    """Restated sharded solve (the library's fmm_plan_set_shard /
    fmm_evaluate_stage): ``stage(s, Q, U)`` for s = 0, 1, 2; between them the
    caller sums ``buffers(0)`` (every level's moments) and then ``buffers(1)``
    (every level's locals) over the shards.  U is accumulated with this
    shard's points' results."""

    def __init__(self, tree: Tree, p: int, ncomp: int = 1, gradient: bool = False):
        self.tree = tree
        self._h = lib().oracle_eval_create(tree._h, p, 1 if gradient else 0, ncomp)
        if not self._h:
            raise ValueError("oracle_eval_create rejected its arguments")

    def set_shard(self, index: int, count: int):
        if lib().oracle_eval_set_shard(self._h, index, count) != 0:
            raise ValueError("bad shard")
        return self

    def stage(self, s: int, Q, U):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        assert U.flags.c_contiguous and U.dtype == np.float64
        if lib().oracle_eval_stage(self._h, s, _dp(Q), _dp(U)) != 0:
            raise ValueError("bad stage")

    def buffers(self, which: int):
        """Per level, a numpy view (no copy) of the moments (0) or locals (1)."""
        out = []
        for level in range(self.tree.depth + 1):
            cnt = C.c_int64()
            ptr = lib().oracle_eval_buffer(self._h, which, level, C.byref(cnt))
            if cnt.value and ptr:
                out.append(np.ctypeslib.as_array(ptr, shape=(cnt.value,)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().oracle_eval_free(h)
            self._h = None
