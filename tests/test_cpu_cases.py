"""The synthetic workloads the bench and the GPU tests run, checked on the host: each
generator's stated definition (extents, topology, jump conditions, stretching, isentropic
relation) holds for the arrays it returns, on sizes that take a fraction of a second."""
import math

import numpy as np
import pytest

from nuc3d_b200 import cases as C


@pytest.mark.parametrize("total,parts,seed", [(1024, 4, 5), (256, 2, 6), (128, 2, 7), (200, 3, 1)])
def test_split_sizes_sum_and_quantum(total, parts, seed):
    n = C.split_sizes(total, parts, seed)
    assert len(n) == parts and sum(n) == total
    assert all(x >= 4 and x % 4 == 0 for x in n)
    assert n == C.split_sizes(total, parts, seed)  # seeded: the same split every time


def test_block_topology_periodic_neighbours():
    parts = [[8, 12], [16, 8, 20], [12, 12]]
    types, ids = C.block_topology(parts)
    nb = 2 * 3 * 2
    assert len(types) == nb
    for b in range(nb):
        for f in range(6):
            n, g = types[b][f], ids[b][f]
            assert 0 <= n < nb and g == f ^ 1
            assert types[n][g] == b  # the neighbour's opposite face points back


def test_normal_shock_rankine_hugoniot():
    g = 1.4
    for m1 in (1.2, 1.5, 3.0):
        r, ur, pr = C.normal_shock(m1, g)
        rho1, u1, p1 = 1.0, m1 * math.sqrt(g), 1.0  # c1 = 1
        rho2, u2, p2 = r * rho1, ur * u1, pr * p1
        # mass, momentum and total enthalpy are continuous across the shock
        assert rho1 * u1 == pytest.approx(rho2 * u2, rel=1e-13)
        assert p1 + rho1 * u1 ** 2 == pytest.approx(p2 + rho2 * u2 ** 2, rel=1e-13)
        h = lambda p, rho, u: g / (g - 1.0) * p / rho + 0.5 * u * u  # noqa: E731
        assert h(p1, rho1, u1) == pytest.approx(h(p2, rho2, u2), rel=1e-13)
        # the downstream flow is subsonic
        assert u2 / math.sqrt(g * p2 / rho2) < 1.0


def test_shock_turbulence_state_and_position():
    shape = (64, 32, 16)
    prim, re, inlet, (X, Y, Z) = C.shock_turbulence(shape, m1=1.5, seed=3)
    nx, ny, nz = shape
    assert prim.shape == (5, nz, ny, nx) and X.shape == (nz + 1, ny + 1, nx + 1)
    h = 2.0 * math.pi / ny
    assert np.allclose(np.diff(X[0, 0]), h) and np.allclose(np.diff(Y[0, :, 0]), h)
    r, ur, pr = C.normal_shock(1.5)
    xc = (np.arange(nx) + 0.5) * h
    up = xc < 0.5 * math.pi
    assert np.all(prim[0][..., up] == 1.0) and np.allclose(prim[0][..., ~up], r)
    assert np.allclose(prim[4][..., ~up] / prim[4][..., up].mean(), pr)
    # the fluctuation rides on the mean velocity m1/mt upstream, ur times it downstream
    assert prim[1][..., up].mean() == pytest.approx(1.5 / 0.6, rel=0.05)
    assert inlet[1] == pytest.approx(1.5 / 0.6) and inlet[4] == pytest.approx(1.0 / (1.4 * 0.36))
    assert re > 0.0
    # the shock locator finds the jump within a cell
    assert abs(C.shock_position(prim[0], h) - 0.5 * math.pi) <= h
    types, ids = C.shock_faces()
    assert types[:2] == [-1, -1] and ids[:2] == [0, 1]


def test_boundary_layer_mesh_state_and_faces():
    shape, nblocks = (64, 32, 16), (4, 2, 2)
    blocks, types, ids, values, params = C.boundary_layer(shape, nblocks, seed=5)
    assert len(blocks) == 16
    assert sum(b["shape"][0] for b in blocks[:4]) == 64
    for b in blocks:
        nx, ny, nz = b["shape"]
        assert nx % 4 == 0 and ny % 4 == 0 and nz % 4 == 0  # block::getJacobians tiles
        X, Y, Z = b["nodes"]
        assert X.shape == Y.shape == Z.shape == (nz + 1, ny + 1, nx + 1)
        # wall-normal spacing grows away from the wall (tanh clustering)
        dy = np.diff(Y[0, :, 0])
        assert np.all(dy > 0.0)
        if b["lo"][1] == 0:
            assert dy[0] < dy[-1]
        rho, u, v, w, p = b["prim"]
        assert np.all(rho > 0.0) and np.all(p > 0.0) and np.all(v == 0.0) and np.all(w == 0.0)
        assert np.all((u >= 0.0) & (u <= 1.0))
    # the bump: the wall rises to h = 0.5 delta at x = 12 delta
    Yw = np.concatenate([b["nodes"][1][0, 0, :-1] for b in blocks[:4]] + [blocks[3]["nodes"][1][0, 0, -1:]])
    Xw = np.concatenate([b["nodes"][0][0, 0, :-1] for b in blocks[:4]] + [blocks[3]["nodes"][0][0, 0, -1:]])
    assert Yw.max() == pytest.approx(0.5, rel=1e-2) and Xw[np.argmax(Yw)] == pytest.approx(12.0, abs=0.5)
    # faces: inlet x-, outlet x+, isothermal wall y-, outlet y+, periodic z
    for k, b in enumerate(blocks):
        a, bb, c = k % 4, (k // 4) % 2, k // 8
        if a == 0:
            assert types[k][0] == -1 and ids[k][0] == 0
            assert np.allclose(values[k][0], [1.0, 1.0, 0.0, 0.0, 1.0 / (1.4 * params["Mach"] ** 2)], rtol=1e-15)
        if a == 3:
            assert types[k][1] == -1 and ids[k][1] == 1
        if bb == 0:
            assert types[k][2] == -1 and ids[k][2] == 2
        if bb == 1:
            assert types[k][3] == -1 and ids[k][3] == 1
        assert types[k][4] >= 0 and types[k][5] >= 0
    assert params["T_wall"] == 1.9 and params["Mach"] == 2.25
    # the wall-adjacent cells sit near the wall temperature (T = gamma Ma^2 p / rho)
    b0 = blocks[0]
    T = 1.4 * 2.25 ** 2 * b0["prim"][4] / b0["prim"][0]
    assert abs(T[:, 0, :].mean() - 1.9) < abs(T[:, -1, :].mean() - 1.9)


def test_gaussian_pulse_isentropic():
    q, m = C.gaussian_pulse((16, 16, 16), amp=0.5)
    # the returned state is U/J; with the uniform box's metrics, rho and p obey p = rho^g/g
    jac = m["jac"]
    rho = q[0] * jac
    E = q[4] * jac
    assert np.allclose(q[1:4], 0.0)
    p = (1.4 - 1.0) * E
    assert np.allclose(p, rho ** 1.4 / 1.4, rtol=1e-13)
    assert rho.max() <= 1.5 and rho.min() >= 1.0
