"""Flow diagnostics (postproc::solveQ: vorticity, enstrophy, Q criterion, kinetic energy)
on the GPU against the reference.

The reference runs block::Post after the golden cases' n steps (tests/golden/diag/);
the GPU evaluates the same state.  The reference-order build must give the same totals
and fields bit for bit, also when the Taylor-Green case is two blocks (the reference run
as two ranks: block sums added in rank order).  The throughput build sums in another
fixed order and may contract to FMA: totals within 1e-12, fields within 1e-11 of their
largest magnitude.
"""
import numpy as np
import pytest

from tests import golden_cases as G


def _state_solver(g, exact):
    s = G.solver(g, exact=exact)
    s.set_q(0, g.qn)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("name", G.diag_names())
def test_diag_bitwise(name):
    g, d = G.load(name), G.load_diag(name)
    s = _state_solver(g, True)
    ens, kin = s.diagnostics()
    assert ens == d["enstrophy"][0] and kin == d["kinetic"][0], (ens - d["enstrophy"][0], kin - d["kinetic"][0])
    f = s.get_diag(0)
    assert np.array_equal(f, d["fields"]), float(np.max(np.abs(f - d["fields"])))
    # a second call on the same state gives the same bits (the workspace is reused)
    assert s.diagnostics() == (ens, kin)


@pytest.mark.gpu
@pytest.mark.parametrize("name", G.diag_names())
def test_diag_fast_roundoff(name):
    g, d = G.load(name), G.load_diag(name)
    s = _state_solver(g, False)
    ens, kin = s.diagnostics()
    assert abs(ens - d["enstrophy"][0]) <= 1e-12 * abs(d["enstrophy"][0])
    assert abs(kin - d["kinetic"][0]) <= 1e-12 * abs(d["kinetic"][0])
    f = s.get_diag(0)
    for c in range(5):
        scale = np.max(np.abs(d["fields"][c]))
        assert np.max(np.abs(f[c] - d["fields"][c])) <= 1e-11 * scale, c


@pytest.mark.gpu
def test_diag_two_blocks_bitwise():
    import nuc3d_b200 as nb
    g, d = G.load("tgv_ns_weno5js_lf"), G.load_diag("tgv_ns_weno5js_lf.2ranks")
    nx, ny, nz = g.cfg["shape"]
    h = nx // 2
    s = nb.Solver(G.nuc3d_config(g, True))
    x, y, z = G.nodes(g)
    for b in range(2):
        s.add_block(h, ny, nz, G.TWO_BLOCK_TYPES[b], G.TWO_BLOCK_IDS[b])
    for b, sl in enumerate((slice(0, h + 1), slice(h, nx + 1))):
        s.set_mesh(b, x[:, :, sl], y[:, :, sl], z[:, :, sl])
    s.finalize()
    left, right = G.split_xi([g.qn], h)
    s.set_q(0, np.ascontiguousarray(left[0]))
    s.set_q(1, np.ascontiguousarray(right[0]))
    ens, kin = s.diagnostics()
    assert ens == d["enstrophy"][0] and kin == d["kinetic"][0]
    assert np.array_equal(np.concatenate([s.get_diag(0), s.get_diag(1)], axis=-1), d["fields"])


@pytest.mark.gpu
def test_diag_taylor_green_initial_energy():
    """At t = 0 the Taylor-Green field has mean kinetic energy 1/8 per cell (rho = 1,
    <u^2 + v^2>/2 over the periodic cell centres); enstrophy 3/8 per cell (|w|^2 mean 3/4)
    up to the sixth-order truncation of the velocity gradients."""
    g = G.load("tgv_ns_weno5js_lf")
    s = G.solver(g, exact=False)
    n = int(np.prod(g.cfg["shape"]))
    ens, kin = s.diagnostics()
    assert abs(kin / n - 0.125) < 1e-12
    assert abs(ens / n - 0.375) < 5e-3


@pytest.mark.gpu
def test_diag_refuses_undefined_gradient_stencil():
    """weno3js (bufferSize 2) with the default cd6 gradients: the reference's diagnostics
    read outside its rows, so the library refuses with NUC3D_ENOTSUP."""
    import nuc3d_b200 as nb
    s = G.solver(G.load("weno3js_euler_lf_bc"), exact=True)
    with pytest.raises(nb.Nuc3dError) as e:
        s.diagnostics()
    assert e.value.code == 5
