"""Grid metrics of a block from its node coordinates, as block::getJacobians does it.

The reference reconstructs cell centres and the covariant derivatives
x_xi ... z_zeta with 5-node Lagrange polynomials over tiles of 4x4x4 cells
(src/block.cpp:147-235 interpolation_lag, :327-477 interpolation_derlag,
coefficients src/block.h:36-48, TILE_SIZE 4 src/block.h:28), then inverts the
3x3 Jacobian per cell (src/block.cpp:237-325).  The sums below run in the
reference's order (xi innermost, then eta, then zeta, each from 0.0), and the
per-cell algebra is written as in getJacobians, so the results are bitwise the
reference's on any IEEE machine.
"""
from __future__ import annotations

import numpy as np

TILE = 4
# src/block.h:36-48
LAG = np.array([
    [35.0 / 128.0, 35.0 / 32.0, -35.0 / 64.0, 7.0 / 32.0, -5.0 / 128.0],
    [-5.0 / 128.0, 15.0 / 32.0, 45.0 / 64.0, -5.0 / 32.0, 3.0 / 128.0],
    [3.0 / 128.0, -5.0 / 32.0, 45.0 / 64.0, 15.0 / 32.0, -5.0 / 128.0],
    [-5.0 / 128.0, 7.0 / 32.0, -35.0 / 64.0, 35.0 / 32.0, 35.0 / 128.0],
])
DERLAG = np.array([
    [-11.0 / 12.0, 17.0 / 24.0, 3.0 / 8.0, -5.0 / 24.0, 1.0 / 24.0],
    [1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0, 0.0],
    [0.0, 1.0 / 24.0, -9.0 / 8.0, 9.0 / 8.0, -1.0 / 24.0],
    [-1.0 / 24.0, 5.0 / 24.0, -3.0 / 8.0, -17.0 / 24.0, 11.0 / 12.0],
])


def _tile_sum(f: np.ndarray, cx: np.ndarray, cy: np.ndarray, cz: np.ndarray) -> np.ndarray:
    """sum_k cz * (sum_j cy * (sum_i cx * f)) over the 5x5x5 nodes of each cell's tile."""
    nz0, ny0, nx0 = f.shape
    nx, ny, nz = nx0 - 1, ny0 - 1, nz0 - 1
    I, J, K = np.arange(nx), np.arange(ny), np.arange(nz)
    ti, tj, tk = (I // TILE) * TILE, (J // TILE) * TILE, (K // TILE) * TILE
    ai, aj, ak = I % TILE, J % TILE, K % TILE
    vz = np.zeros((nz, ny, nx))
    for k in range(5):
        vy = np.zeros((nz, ny, nx))
        for j in range(5):
            vx = np.zeros((nz, ny, nx))
            sub = f[(tk + k)[:, None], (tj + j)[None, :], :]
            for i in range(5):
                vx = vx + cx[ai, i][None, None, :] * sub[:, :, ti + i]
            vy = vy + cy[aj, j][None, :, None] * vx
        vz = vz + cz[ak, k][:, None, None] * vy
    return vz


def metrics_from_nodes(x, y, z) -> dict:
    """x, y, z: node coordinates shaped (nz+1, ny+1, nx+1); cells multiple of 4 per axis.

    Returns jac (N), xi_xyz/eta_xyz/zeta_xyz (3, nz, ny, nx), dxyz (9, nz, ny, nx) ordered
    x_xi x_eta x_zeta y_xi y_eta y_zeta z_xi z_eta z_zeta, and xyz_center (3, nz, ny, nx).
    """
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    for n in x.shape:
        if (n - 1) % TILE or n < TILE + 1:
            raise ValueError("the reference's tile-Lagrange metrics need cells per axis "
                             f"to be a multiple of {TILE} (node dims {x.shape[::-1]})")
    der = [(DERLAG, LAG, LAG), (LAG, DERLAG, LAG), (LAG, LAG, DERLAG)]
    # dx[d], dy[d], dz[d] = d(x, y, z)/d(xi_d)   (src/block.cpp:251-256)
    dx = [_tile_sum(x, *der[d]) for d in range(3)]
    dy = [_tile_sum(y, *der[d]) for d in range(3)]
    dz = [_tile_sum(z, *der[d]) for d in range(3)]
    x_xi, x_eta, x_zeta = dx
    y_xi, y_eta, y_zeta = dy
    z_xi, z_eta, z_zeta = dz
    # src/block.cpp:285-300
    jacob = 1.0 / (x_xi * (y_eta * z_zeta - y_zeta * z_eta)
                   + x_eta * (y_zeta * z_xi - y_xi * z_zeta)
                   + x_zeta * (y_xi * z_eta - y_eta * z_xi))
    if np.any(jacob < 0.0):
        raise ValueError("negative Jacobian (the reference exits here, src/block.cpp:314-318)")
    xi = np.stack([(y_eta * z_zeta - y_zeta * z_eta) * jacob,
                   (x_zeta * z_eta - x_eta * z_zeta) * jacob,
                   (x_eta * y_zeta - x_zeta * y_eta) * jacob])
    eta = np.stack([(y_zeta * z_xi - y_xi * z_zeta) * jacob,
                    (x_xi * z_zeta - x_zeta * z_xi) * jacob,
                    (x_zeta * y_xi - x_xi * y_zeta) * jacob])
    zeta = np.stack([(y_xi * z_eta - y_eta * z_xi) * jacob,
                     (x_eta * z_xi - x_xi * z_eta) * jacob,
                     (x_xi * y_eta - x_eta * y_xi) * jacob])
    centre = np.stack([_tile_sum(a, LAG, LAG, LAG) for a in (x, y, z)])
    return {
        "jac": jacob, "xi_xyz": xi, "eta_xyz": eta, "zeta_xyz": zeta,
        "dxyz": np.stack([x_xi, x_eta, x_zeta, y_xi, y_eta, y_zeta, z_xi, z_eta, z_zeta]),
        "xyz_center": centre,
    }
