import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_cases():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    d = {k: z[k] for k in z.files}
    n, seed, p, max_level, ppn, va, flags, qdim = (int(x) for x in d["meta"])
    d.update(n=n, seed=seed, p=p, max_level=max_level, max_ppn=ppn, vertical_axis=va, flags=flags,
             qdim=qdim, phideg=float(d["phideg"][0]))
    if "FIELD" in d:
        d["FIELD"] = d["FIELD"].reshape(-1, 3)
    for k in ("VECPOT", "BIOT"):
        if k in d:
            d[k] = d[k].reshape(-1, 3)
    return d


def golden_tree(sf, g, ctx):
    """The library's tree for a golden case (explicit root cube if the case has one)."""
    box = (g["box_corner"], float(g["box_width"][0])) if "box_corner" in g else None
    return sf.Tree(g["pos"], g["max_level"], g["max_ppn"], g["vertical_axis"], g["phideg"], ctx=ctx, box=box)


def golden_exclusions(g):
    """(row_ptr, cols, near_too) of a case's self_generator {i, i+s1, i+s2}, or None."""
    if "strides" not in g:
        return None
    n = g["n"]
    s1, s2 = (int(x) for x in g["strides"])
    i = np.arange(n)
    cols = np.stack([i, (i + s1) % n, (i + s2) % n], axis=1).reshape(-1).astype(np.int32)
    row_ptr = np.arange(0, 3 * n + 1, 3, dtype=np.int64)
    near_too = bool(g["flags"] & 128)
    return row_ptr, cols, near_too


TREE_KEYS = ("CNODE", "ILEAF", "IDXP", "IDXV", "ILP", "ILV", "CLP", "CLV", "PL", "NLP", "NLV")


def tree_keys(d):
    return sorted(k for k in d if k.startswith(TREE_KEYS) or k == "PARTS")


def rel_err_per_target(got, ref, scale=None, floor_frac=1e-3):
    """Largest per-target relative error.

    With ``scale`` (per-target magnitude sums S_i = sum_j |Q_j|/r_ij for a
    potential, sum_j |Q_j|/r_ij^2 for a field) it is max_i |got_i - ref_i| / S_i:
    the error relative to the size of the terms summed at target i, which is
    what FP64 rounding is proportional to (a sum of +-q/r can cancel to almost
    nothing, where |ref_i| is no meaningful denominator).  Without ``scale``
    the denominator is max(|ref_i|, floor_frac * RMS|ref|)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.ndim == 2:
        d = np.linalg.norm(got - ref, axis=1)
        r = np.linalg.norm(ref, axis=1)
    else:
        d = np.abs(got - ref)
        r = np.abs(ref)
    if not r.size:
        return 0.0
    if scale is not None:
        return float(np.max(d / np.asarray(scale, dtype=np.float64)))
    floor = floor_frac * np.sqrt(np.mean(r * r))
    return float(np.max(d / np.maximum(r, floor)))


def rel_l2(got, ref):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


@pytest.fixture(scope="session")
def golden():
    return load_golden
