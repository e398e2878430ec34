"""Synthetic workloads with the shapes of the reference's benchmark configurations.

No dataset is involved: every state is generated from a formula.
  * taylor_green     -- block::initial_taylorgreen (src/block.cpp:683-690), periodic box
  * spherical_riemann-- rho, p = 1, 10 for r < 0.2 and 0.125, 0.1 outside, u = 0,
                        outlet (extrapolation) faces; the reference has no initialiser
                        for it, so the state is injected like its restart file
                        (src/block.cpp:785-816)
Uniform boxes get analytic metrics (xi_x = 1/hx, jac = 1/(hx hy hz)); curvilinear
meshes go through nuc3d_b200.metrics (block::getJacobians).
"""
from __future__ import annotations

import math

import numpy as np

PERIODIC_NEIGHBOUR_FACE = (1, 0, 3, 2, 5, 4)


def uniform_metrics(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)) -> dict:
    nx, ny, nz = shape
    h = [(hi[d] - lo[d]) / n for d, n in enumerate(shape)]
    N = (nz, ny, nx)
    one = np.ones(N)
    zero = np.zeros(N)
    jac = one / (h[0] * h[1] * h[2])
    return {
        "jac": jac,
        "xi_xyz": np.stack([one / h[0], zero, zero]),
        "eta_xyz": np.stack([zero, one / h[1], zero]),
        "zeta_xyz": np.stack([zero, zero, one / h[2]]),
        "dxyz": np.stack([one * h[0], zero, zero, zero, one * h[1], zero, zero, zero, one * h[2]]),
    }


def centres(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    nx, ny, nz = shape
    c = [lo[d] + (np.arange(n) + 0.5) * (hi[d] - lo[d]) / n for d, n in enumerate(shape)]
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    return X, Y, Z


def prim_to_q(prim, jac, gamma):
    """U/J with the arithmetic of block::initialQ (src/block.cpp:554-563)."""
    rho, u, v, w, p = prim
    rhoe = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho / jac, (rho * u) / jac, (rho * v) / jac, (rho * w) / jac, rhoe / jac])


def spherical_riemann(shape, gamma=1.4, radius=0.2):
    X, Y, Z = centres(shape)
    r2 = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2
    inside = r2 < radius * radius
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 10.0, 0.1)
    zero = np.zeros_like(rho)
    m = uniform_metrics(shape)
    return prim_to_q(np.stack([rho, zero, zero, zero, p]), m["jac"], gamma), m


def taylor_green(shape, gamma=1.4, mach=0.1):
    lo, hi = (0.0,) * 3, (2.0 * math.pi,) * 3
    X, Y, Z = centres(shape, lo, hi)
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    rho = np.ones_like(u)
    p = 1.0 / (gamma * mach * mach) + ((np.cos(2.0 * Z) + 2.0) * (np.cos(2.0 * X) + np.cos(2.0 * Y)) - 2.0) / 16.0
    m = uniform_metrics(shape, lo, hi)
    return prim_to_q(np.stack([rho, u, v, w, p]), m["jac"], gamma), m


def outlet_faces():
    return [-1] * 6, [1] * 6


def periodic_faces(block=0):
    return [block] * 6, list(PERIODIC_NEIGHBOUR_FACE)
