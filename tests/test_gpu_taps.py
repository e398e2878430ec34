"""Debug taps (nuc3d_debug_get) against the reference's own intermediates: the taps harness
runs one right-hand side of the reference on a golden case's state and dumps every
direction's EulerFlux members (split fluxes FluxL/FluxR, reconstructions
reconstFluxL/reconstFluxR) and flux differences (dfdxi, dgdeta, dhdzeta); the
reference-order build's taps must equal them bit for bit.  Cases cover every explicit
scheme, the compact schemes (rows + Thomas), all four physical BC types, periodic faces
and curvilinear metrics."""
import numpy as np
import pytest

from oracle import refrun as R
from tests import golden_cases as G

CASES = ["sphere_euler_weno5z_ausm_outlet", "bc_ns_weno7js_ausmp", "mixed_low_order_ausmp",
         "wavy_euler_weno5js_lf", "mixed_compact_ausmp", "mixed_hccs77_euler_ausmp",
         "ns_ausm_weno5z_wall_inlet"]
DIRS = ("xi", "eta", "zeta")
DF = ("dfdxi", "dgdeta", "dhdzeta")


def _reference_rhs(g):
    p = g.cfg["params"]
    values = [G.inlet_state(p) if k == "inlet" else None for k in g.cfg["faces"]]
    case = R.Case(model=g.cfg["model"], riemann=g.cfg["riemann"], schemes=tuple(g.cfg["schemes"]),
                  vis=G.vis(g), params=p, nodes=[G.nodes(g)],
                  bc_topo=[R.bc_lines(g.cfg["faces"], values)], q0=[g.q0], start_step=1)
    return R.run(case, "rhs", timeout=600)[0]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_taps_bitwise(name):
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    g = G.load(name)
    ref = _reference_rhs(g)
    s = G.solver(g, exact=True)
    status0, resets0 = s.status(), s.energy_resets()
    for d, dn in enumerate(DIRS):
        for kind, key in (("FluxL", f"FluxL_{dn}"), ("FluxR", f"FluxR_{dn}"),
                          ("rFluxL", f"rFluxL_{dn}"), ("rFluxR", f"rFluxR_{dn}"), ("df", DF[d])):
            got = s.debug_get(0, kind, d)
            want = R.stack(ref, key, 5)
            assert got.shape == want.shape, (kind, dn, got.shape, want.shape)
            if not np.array_equal(got, want):
                bad = np.argwhere(got != want)
                raise AssertionError(f"{name} {kind} {dn}: {len(bad)} values differ, first "
                                     f"{bad[:4].tolist()}, max |diff| "
                                     f"{float(np.max(np.abs(got - want))):.3g}")
    assert s.status() == status0 and s.energy_resets() == resets0
    # the taps' differences are the right-hand side's inviscid part: their sum is the
    # Euler RHS (NS: minus the viscous part)
    if g.cfg["model"] == "Euler3d":
        s.rhs()
        rhs = s.get_rhs(0)
        df = [s.debug_get(0, "df", d) for d in range(3)]
        tot = df[0] + np.transpose(df[1], (0, 2, 3, 1)) + np.transpose(df[2], (0, 3, 1, 2))
        assert np.allclose(tot, rhs, rtol=1e-12, atol=1e-12 * np.abs(rhs).max())
    s.close()


@pytest.mark.gpu
def test_taps_throughput_build():
    """The throughput build's taps agree with the reference-order build's to round-off."""
    g = G.load("sphere_euler_weno5z_ausm_outlet")
    a, b = G.solver(g, exact=True), G.solver(g, exact=False)
    for d in range(3):
        for kind in a.TAP_KINDS:
            x, y = a.debug_get(0, kind, d), b.debug_get(0, kind, d)
            assert np.max(np.abs(x - y)) <= 1e-12 * max(np.max(np.abs(x)), 1e-300), (kind, d)
    a.close()
    b.close()
