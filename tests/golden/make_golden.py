"""Generate the golden fixtures from the compiled reference.

Run in a container that has the reference checkout (``make -C oracle ref``
first).  Each case is a seeded synthetic input; the fixture stores the inputs
and everything the reference's driver dumped (tree, lists, U), so tests on a
machine without the reference still compare against the reference's own
output.  ``python tests/golden/make_golden.py`` rewrites every ``*.npz`` here.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import refio  # noqa: E402
from simplefmm_b200 import workloads as W  # noqa: E402

HERE = Path(__file__).resolve().parent

T, POT, FIELD, VEC, BIOT = refio.FLAG_TREE, refio.FLAG_POT, refio.FLAG_FIELD, refio.FLAG_VECPOT, refio.FLAG_BIOT

# name: (distribution, n, seed, p, max_level, max_ppn, vertical_axis, phideg, flags, charge kind, qdim)
CASES = {
    "uniform_n3000_p6": ("uniform", 3000, 11, 6, 20, 64, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "plummer_n6000_p5_ppn32": ("plummer", 6000, 12, 5, 20, 32, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "shell_n4000_p4_ppn16": ("shell", 4000, 13, 4, 20, 16, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "gauss2_n4000_p8": ("gauss2", 4000, 14, 8, 20, 64, 2, 0.0, T | POT | FIELD, "sign", 1),
    "uniform_n2500_p10_maxlevel3": ("uniform", 2500, 15, 10, 3, 8, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "uniform_n60_p4_single_leaf": ("uniform", 60, 16, 4, 20, 64, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "uniform_n400_p4_depth1": ("uniform", 400, 17, 4, 20, 64, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "vector_n2000_p8_ppn128": ("uniform", 2000, 18, 8, 20, 128, 2, 0.0, T | VEC | BIOT, "uniform", 3),
    "axis0_n3000_p6": ("plummer", 3000, 19, 6, 20, 32, 0, 0.0, T | POT, "uniform", 1),
    "phi30_n3000_p6": ("uniform", 3000, 20, 6, 20, 32, 2, 30.0, T | POT, "uniform", 1),
    "uniform_n3000_p12": ("uniform", 3000, 21, 12, 20, 64, 2, 0.0, POT | FIELD, "uniform", 1),
    "uniform_n3000_p13": ("uniform", 3000, 25, 13, 20, 64, 2, 0.0, POT | FIELD, "uniform", 1),
    "plummer_n3000_p16_ppn32": ("plummer", 3000, 26, 16, 20, 32, 2, 0.0, T | POT | FIELD, "uniform", 1),
    "box_n3000_p6": ("uniform", 3000, 22, 6, 20, 64, 2, 0.0, T | POT | FIELD | refio.FLAG_BOX, "uniform", 1),
    "exclude_n3000_p6": ("plummer", 3000, 23, 6, 20, 32, 2, 0.0, POT | FIELD | refio.FLAG_EXCLUDE, "uniform", 1),
    "exclude_far_n3000_p6": ("plummer", 3000, 24, 6, 20, 32, 2, 0.0, POT | FIELD | refio.FLAG_EXCLUDE_FAR,
                             "uniform", 1),
}

# cases run by the reference built with its dense-M2L option (-DFMM_M2L_DIRECT)
DIRECT = {"direct_plummer_n4000_p8": ("plummer", 4000, 27, 8, 20, 32, 2, 0.0, POT | FIELD, "uniform", 1),
          "direct_vector_n2000_p6": ("uniform", 2000, 28, 6, 20, 64, 2, 0.0, VEC | BIOT, "uniform", 3)}
CASES.update(DIRECT)

# explicit root cube (corner, width) and exclusion strides of the cases above
BOXES = {"box_n3000_p6": ((-0.25, -0.5, -0.125), 2.0)}
STRIDES = {"exclude_n3000_p6": (1, 1777), "exclude_far_n3000_p6": (1, 1777)}


def make_case(name, spec):
    dist, n, seed, p, max_level, ppn, va, phideg, flags, qkind, qdim = spec
    pos = W.points(dist, n, seed)
    q = W.charges(n, seed, qkind, qdim)
    out = refio.run_reference(pos, q, p=p, max_level=max_level, max_ppn=ppn, vertical_axis=va,
                              phideg=phideg, flags=flags, native=True, box=BOXES.get(name), strides=STRIDES.get(name),
                              direct=name in DIRECT)
    arrays = {k: v for k, v in out.items() if not k.startswith("T_")}
    if name in BOXES:
        arrays["box_corner"] = np.array(BOXES[name][0])
        arrays["box_width"] = np.array([BOXES[name][1]])
    if name in STRIDES:
        arrays["strides"] = np.array(STRIDES[name])
    meta = np.array([n, seed, p, max_level, ppn, va, flags, qdim], dtype=np.int64)
    if name in DIRECT:
        arrays["m2l_direct"] = np.array([1])
    np.savez_compressed(HERE / f"{name}.npz", pos=pos, q=q, meta=meta, phideg=np.array([phideg]),
                        dist=np.array([dist]), **arrays)


def main():
    if not refio.have_reference(native=True):
        sys.exit("oracle/_ref/ref_driver_native is not built (make -C oracle ref)")
    only = set(sys.argv[1:])
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        make_case(name, spec)
        print("wrote", name)


if __name__ == "__main__":
    main()
