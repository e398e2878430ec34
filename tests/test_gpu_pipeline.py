"""The pipelined sweeps (persistent kernels fed by tensor-map loads, sweep_pipe.cuh) give
exactly what the one-tile-per-CTA sweeps give, which the parity tests pin to the
reference: right-hand side, dt and steps on every explicit-scheme golden case, Euler and
Navier-Stokes (the viscous fluxes loaded by the consumers, the viscous differences in
phase 3), with every tile shape, across block faces (two blocks), with the energy reset,
and in both builds."""
import numpy as np
import pytest

from tests import golden_cases as G

EXPLICIT = [n for n in G.names()
            if not any(s in ("crweno5", "hccs", "hccs77") for s in G.load(n).cfg["schemes"])]


def _run(g, exact, pipe, shape=None, nsteps=None):
    s = G.solver(g, exact=exact)
    s.set_pipeline(pipe)
    assert bool(s.pipeline()) == pipe
    if shape is not None:
        s.set_tiles(shape)
    dt = s.rhs()
    rhs = s.get_rhs(0)
    s.step(int(nsteps or g.cfg["nsteps"]))
    out = dt, rhs, s.get_q(0), s.time_dt(), s.energy_resets(), s.status(), s.residual()
    s.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXPLICIT)
def test_pipelined_sweeps_bitwise_reference(name):
    g = G.load(name)
    dt, rhs, q, (t, dtl), resets, _, res = _run(g, exact=True, pipe=True)
    assert dt == g.dt_local[0]
    assert np.array_equal(rhs, g.rhs)
    assert np.array_equal(q, g.qn)
    assert dtl == g.dt[-1] and t == g.time[-1]
    assert res == g.res[-1]


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere_euler_weno5z_ausm_outlet", "mixed_euler_lf_outlet_symm",
                                  "sphere_reset_euler_weno5z_ausm", "mixed_low_order_ausmp",
                                  "tgv_ns_weno5js_lf", "bc_ns_weno7js_ausmp", "ns_cd8_weno7js_lf"])
@pytest.mark.parametrize("shape", [(0, 0, 0), (1, 1, 1), (2, 2, 2), (2, 0, 1)])
@pytest.mark.parametrize("exact", [True, False])
def test_pipelined_equals_plain(name, shape, exact):
    """Reference-order build: identical bits.  Throughput build: the compiler contracts
    multiply-adds into FMAs per kernel, so the two kernels agree to round-off (the parity
    tests' relative max-norm 1e-11)."""
    g = G.load(name)
    a = _run(g, exact, True, shape)
    b = _run(g, exact, False, shape)
    if exact:
        assert a[0] == b[0]
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(a[2], b[2])
        assert a[3] == b[3] and a[4] == b[4] and a[5] == b[5] and a[6] == b[6]
    else:
        assert abs(a[0] - b[0]) <= 1e-11 * b[0]
        assert _rel(a[1], b[1]) < 1e-11 and _rel(a[2], b[2]) < 1e-11
        assert a[5] == b[5] and abs(a[6] - b[6]) <= 1e-9 * b[6]


@pytest.mark.gpu
def test_pipelined_two_blocks_bitwise():
    """Halo cells across a block face come from the neighbour block (the producer warp's
    gather): two blocks of the wavy periodic case equal the one-block reference."""
    import nuc3d_b200 as nb
    g = G.load("wavy_euler_weno5js_lf")
    nx, ny, nz = g.cfg["shape"]
    x, y, z = G.nodes(g)
    h = nx // 2
    s = nb.Solver(G.nuc3d_config(g, exact=True))
    t0, i0, _ = G.bc_arrays(g, 0)
    t1, i1, _ = G.bc_arrays(g, 1)
    t0[0], i0[0], t0[1], i0[1] = 1, 1, 1, 0
    t1[0], i1[0], t1[1], i1[1] = 0, 1, 0, 0
    b0 = s.add_block(h, ny, nz, t0, i0)
    b1 = s.add_block(nx - h, ny, nz, t1, i1)
    s.set_mesh(b0, x[:, :, :h + 1], y[:, :, :h + 1], z[:, :, :h + 1])
    s.set_mesh(b1, x[:, :, h:], y[:, :, h:], z[:, :, h:])
    s.finalize()
    assert s.pipeline()
    s.set_q(b0, g.q0[:, :, :, :h])
    s.set_q(b1, g.q0[:, :, :, h:])
    s.step(int(g.cfg["nsteps"]))
    q = np.concatenate([s.get_q(b0), s.get_q(b1)], axis=3)
    assert np.array_equal(q, g.qn)


@pytest.mark.gpu
def test_pipeline_applies_where_it_can():
    """Euler and Navier-Stokes contexts run pipelined; a block with an odd nx (rows not
    16-byte multiples) keeps the one-tile-per-CTA sweeps; switching it off and on again
    works, and a mask selects directions."""
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    assert G.solver(G.load("tgv_ns_weno5js_lf"), exact=True).pipeline() == 7
    e = G.solver(G.load("sphere_euler_weno5z_ausm_outlet"), exact=True)
    assert e.pipeline() == 7
    e.set_pipeline(False)
    assert e.pipeline() == 0
    e.set_pipeline(True)
    assert e.pipeline() == 7
    e.set_pipeline(4)
    assert e.pipeline() == 4
    q, m = C.spherical_riemann((13, 12, 12))
    o = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0))
    b = o.add_block(13, 12, 12, *C.outlet_faces())
    o.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    o.finalize()
    assert o.pipeline() == 0
