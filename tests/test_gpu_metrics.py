"""Metrics on the GPU (nuc3d_block_set_nodes) against block::getJacobians.

The device kernel must give the reference's metrics bit for bit: against the metrics the
reference itself dumped for the Taylor-Green fixture, against the host restatement
(nuc3d_b200.metrics, itself pinned to the reference) on every golden mesh and on a
stretched boundary-layer mesh with a bump, and through a right-hand side.
"""
import math

import numpy as np
import pytest

from tests import golden_cases as G


def _device_metrics(shape, nodes, faces=([-1] * 6, [1] * 6)):
    import nuc3d_b200 as nb
    s = nb.Solver(nb.Config())
    b = s.add_block(*shape, *faces)
    s.set_nodes(b, *nodes)
    return s.get_metrics(b)


@pytest.mark.gpu
def test_device_metrics_equal_reference_dump():
    g = G.load("tgv_ns_weno5js_lf")
    m = _device_metrics(g.cfg["shape"], G.nodes(g))
    assert np.array_equal(m["jac"], g.metrics_jac)
    for nm in ("xi_xyz", "eta_xyz", "zeta_xyz"):
        assert np.array_equal(m[nm], g.data[f"metrics_{nm}"]), nm


@pytest.mark.gpu
@pytest.mark.parametrize("name", G.names())
def test_device_metrics_equal_host(name):
    from nuc3d_b200.metrics import metrics_from_nodes
    g = G.load(name)
    nodes = G.nodes(g)
    h, d = metrics_from_nodes(*nodes), _device_metrics(g.cfg["shape"], nodes)
    for k in ("jac", "xi_xyz", "eta_xyz", "zeta_xyz"):
        assert np.array_equal(h[k], d[k]), k


@pytest.mark.gpu
def test_device_metrics_stretched_bump_mesh():
    """Wall-normal tanh stretching and a Gaussian bump (the geometry of the reference's
    boundary-layer configuration, scaled down)."""
    from nuc3d_b200.metrics import metrics_from_nodes
    nx, ny, nz = 64, 32, 16
    xi = np.linspace(0.0, 20.0, nx + 1)
    eta = np.tanh(2.5 * np.linspace(0.0, 1.0, ny + 1)) / math.tanh(2.5) * 3.0
    zz = np.linspace(0.0, 2.0, nz + 1)
    Z, Y, X = np.meshgrid(zz, eta, xi, indexing="ij")
    bump = 0.5 * np.exp(-((X - 10.0) / 2.0) ** 2)
    Y = Y + bump * (1.0 - Y / 3.0)
    h, d = metrics_from_nodes(X, Y, Z), _device_metrics((nx, ny, nz), (X, Y, Z))
    for k in ("jac", "xi_xyz", "eta_xyz", "zeta_xyz"):
        assert np.array_equal(h[k], d[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["wavy_euler_weno5js_lf", "bc_ns_weno7js_ausmp"])
def test_rhs_bitwise_with_device_metrics(name):
    import nuc3d_b200 as nb
    g = G.load(name)
    s = nb.Solver(G.nuc3d_config(g, True))
    t, i, v = G.bc_arrays(g)
    b = s.add_block(*g.cfg["shape"], t, i, v)
    x, y, z = G.nodes(g)
    s.set_nodes(b, x, y, z)
    if any(tt == -1 and ii == 3 for tt, ii in zip(t, i)):   # symmetry faces need dxyz
        from nuc3d_b200.metrics import metrics_from_nodes
        m = metrics_from_nodes(x, y, z)
        s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, g.q0)
    assert s.rhs() == g.dt_local[0]
    assert np.array_equal(s.get_rhs(0), g.rhs)


@pytest.mark.gpu
def test_device_metrics_reject_negative_jacobian():
    import nuc3d_b200 as nb
    from oracle.refrun import box_nodes
    x, y, z = box_nodes(8, 8, 8)
    with pytest.raises(nb.Nuc3dError) as e:
        _device_metrics((8, 8, 8), (x[:, :, ::-1].copy(), y, z))
    assert e.value.code == 1
