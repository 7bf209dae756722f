"""Test-infrastructure helpers around the compiled reference (``oracle/_ref``).

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
use this module: it is a test oracle, never the thing measured or shipped.

``run_reference`` writes an input file in the format ``ref_driver.cpp``
documents, runs the reference binary (optionally as several shim ranks, like
``mpirun -n K``), and parses the sectioned output.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_DIR = ORACLE_DIR / "_ref"

FLAG_TREE = 1
FLAG_POT = 2
FLAG_FIELD = 4
FLAG_VECPOT = 8
FLAG_BIOT = 16
FLAG_TREE_ONLY = 32
FLAG_BOX = 64            # explicit cube: corner (3) and width follow the charges
FLAG_EXCLUDE = 128       # self_generator {i, i+s1, i+s2} with the matching is_self
FLAG_EXCLUDE_FAR = 256   # the same generator, default is_self (only non-neighbours removed)


def ref_binary(native: bool = False, direct: bool = False) -> Path:
    """The compiled reference: portable, -march=native, or -march=native with
    the reference's dense-M2L build option (-DFMM_M2L_DIRECT)."""
    if direct:
        return REF_DIR / "ref_driver_direct"
    return REF_DIR / ("ref_driver_native" if native else "ref_driver")


def have_reference(native: bool = False) -> bool:
    return ref_binary(native).exists()


def write_input(path, pos, q, p, max_level, max_ppn, vertical_axis=2, phideg=0.0, flags=FLAG_POT,
                box=None, strides=None):
    pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    q = np.ascontiguousarray(q, dtype=np.float64)
    qdim = 1 if q.ndim == 1 else q.shape[1]
    with open(path, "wb") as f:
        f.write(b"SFMMIN01")
        f.write(struct.pack("<q4id2i", pos.shape[0], p, max_level, max_ppn, vertical_axis, phideg, qdim, flags))
        f.write(pos.tobytes())
        f.write(q.reshape(-1).tobytes())
        if flags & FLAG_BOX:
            f.write(struct.pack("<4d", box[0][0], box[0][1], box[0][2], box[1]))
        if flags & (FLAG_EXCLUDE | FLAG_EXCLUDE_FAR):
            f.write(struct.pack("<2i", strides[0], strides[1]))


_INT64_TAGS = ("CNODE", "CLV", "PL")


def read_output(path) -> dict:
    data = Path(path).read_bytes()
    assert data[:8] == b"SFMMOUT1", "not a reference output file"
    off = 8
    out = {}
    while off < len(data):
        tag = data[off:off + 8].rstrip(b"\0").decode()
        (nb,) = struct.unpack("<q", data[off + 8:off + 16])
        payload = data[off + 16:off + 16 + nb]
        off += 16 + nb
        if tag.startswith("T_") or tag in ("BOX", "POT", "FIELD", "VECPOT", "BIOT"):
            arr = np.frombuffer(payload, dtype=np.float64).copy()
            out[tag] = float(arr[0]) if tag.startswith("T_") else arr
        elif tag.startswith(_INT64_TAGS) and not tag.startswith("PARTS"):
            out[tag] = np.frombuffer(payload, dtype=np.int64).copy()
        else:
            out[tag] = np.frombuffer(payload, dtype=np.int32).copy()
    if "FIELD" in out:
        out["FIELD"] = out["FIELD"].reshape(-1, 3)
    for k in ("VECPOT", "BIOT"):
        if k in out:
            out[k] = out[k].reshape(-1, 3)
    return out


def run_reference(pos, q, p, max_level=20, max_ppn=64, vertical_axis=2, phideg=0.0,
                  flags=FLAG_POT, ranks=1, native=False, timeout=3600, box=None, strides=None, direct=False) -> dict:
    """Run the compiled reference on (pos, q) and return its parsed output."""
    binary = ref_binary(native, direct)
    if not binary.exists():
        raise FileNotFoundError(f"{binary} is not built (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(fin, pos, q, p, max_level, max_ppn, vertical_axis, phideg, flags, box, strides)
        env = dict(os.environ, SIMPLEFMM_SHIM_NP=str(ranks))
        r = subprocess.run([str(binary), fin, fout], env=env, capture_output=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference failed rc={r.returncode}: {r.stderr.decode()[-2000:]}")
        return read_output(fout)


def tree_levels(out: dict) -> int:
    return int(out["DEPTH"][0])
