"""Seeded synthetic point sets for the benchmark workloads.

The reference ships no datasets (its driver draws ``std::rand`` points in the
unit cube, main.cpp:22-34).  These generators produce the distributions the
benchmark configurations name, from a numpy ``Generator`` seeded explicitly so
every run (GPU path, oracle, reference) sees identical inputs.
"""
from __future__ import annotations

import numpy as np


def uniform_cube(n: int, seed: int) -> np.ndarray:
    """n points uniform in [0, 1]^3."""
    rng = np.random.default_rng(seed)
    return rng.random((n, 3))


def plummer(n: int, seed: int, a: float = 1.0, rmax: float = 10.0) -> np.ndarray:
    """Plummer sphere of scale radius ``a``, radii truncated at ``rmax``.

    Radius by inverse CDF: r = a / sqrt(X^(-2/3) - 1), X ~ U(0, 1]; samples
    with r > rmax are redrawn.  Directions are isotropic.
    """
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while out.shape[0] < n:
        m = int((n - out.shape[0]) * 1.05) + 16
        x = rng.random(m)
        x = np.where(x == 0.0, 0.5, x)
        r = a / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
        ct = rng.uniform(-1.0, 1.0, m)
        ph = rng.uniform(0.0, 2.0 * np.pi, m)
        st = np.sqrt(1.0 - ct * ct)
        pts = np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], axis=1)
        out = np.concatenate([out, pts[r <= rmax]])
    return out[:n]


def thin_shell(n: int, seed: int, radius: float = 1.0, thickness: float = 0.01) -> np.ndarray:
    """Points uniform in volume in the shell radius-thickness/2 .. radius+thickness/2."""
    rng = np.random.default_rng(seed)
    r0, r1 = radius - thickness / 2, radius + thickness / 2
    r = np.cbrt(rng.uniform(r0 ** 3, r1 ** 3, n))
    ct = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    st = np.sqrt(1.0 - ct * ct)
    return np.stack([r * st * np.cos(ph), r * st * np.sin(ph), r * ct], axis=1)


def two_gaussians(n: int, seed: int, sigma: float = 0.05, separation: float = 0.5) -> np.ndarray:
    """Two isotropic Gaussian clusters (n/2 each) centred ``separation`` apart
    along x about the centre of the unit cube, clipped into [0, 1]^3."""
    rng = np.random.default_rng(seed)
    n0 = n // 2
    c0 = np.array([0.5 - separation / 2, 0.5, 0.5])
    c1 = np.array([0.5 + separation / 2, 0.5, 0.5])
    pts = rng.normal(0.0, sigma, (n, 3))
    pts[:n0] += c0
    pts[n0:] += c1
    return np.clip(pts, 0.0, 1.0)


def charges(n: int, seed: int, kind: str = "uniform", dim: int = 1) -> np.ndarray:
    """Charges uniform in [-1, 1] (``kind='uniform'``) or +-1 with equal
    probability (``kind='sign'``); shape (n,) for dim 1 else (n, dim)."""
    rng = np.random.default_rng(seed + 7919)
    shape = (n,) if dim == 1 else (n, dim)
    if kind == "sign":
        return np.where(rng.random(shape) < 0.5, -1.0, 1.0)
    return rng.uniform(-1.0, 1.0, shape)


DISTRIBUTIONS = {
    "uniform": uniform_cube,
    "plummer": plummer,
    "shell": thin_shell,
    "gauss2": two_gaussians,
}


def points(kind: str, n: int, seed: int) -> np.ndarray:
    return DISTRIBUTIONS[kind](n, seed)
