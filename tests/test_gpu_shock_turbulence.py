"""The shock-turbulence workload (a Mach 1.5 normal shock in the 24-block case's decaying
turbulence: inflow through x-, outflow through x+, periodic y and z; Navier-Stokes,
WENO5-Z, AUSM, cd6) against the reference itself, at a reduced size (64 x 32 x 32) so that
the reference runs in seconds: the inlet face's BC values (src/boundaryConditions.cpp:
140-274), the outlet's extrapolation (:307-459) and the periodic faces all act.  The
reference-order build must reproduce the state and every dt bit for bit after 3 steps; the
throughput build within 1e-11 relative max-norm."""
import numpy as np
import pytest

from oracle import refrun as R

SHAPE, STEPS = (64, 32, 32), 3


def _setup():
    from nuc3d_b200 import cases as C
    prim, re, inlet, (x, y, z) = C.shock_turbulence(SHAPE)
    h = 2.0 * np.pi / SHAPE[1]
    q0 = C.prim_to_q(prim, np.full(prim.shape[1:], 1.0 / (h * h * h)), 1.4)
    return C, q0, re, inlet, (x, y, z)


@pytest.fixture(scope="module")
def ref():
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    C, q0, re, inlet, nodes = _setup()
    topo = ["-1 0 " + " ".join(repr(float(v)) for v in inlet), "-1 1", "0 3", "0 2", "0 5", "0 4"]
    case = R.Case(model="NavierStokes3d", riemann="AUSM", schemes=("weno5z",) * 3,
                  params={"Reynolds": re, "Mach": 0.6, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
                          "T_inf": 288.0, "T_wall": 1.0},
                  nodes=[nodes], bc_topo=[topo], q0=[q0], start_step=1)
    out = R.run(case, "steps", STEPS, timeout=1200)[0]
    return R.stack(out, "Q", 5), out["dt"], out["time"], out["res"]


def _gpu(exact):
    import nuc3d_b200 as nb
    C, q0, re, inlet, nodes = _setup()
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                            reynolds=re, mach=0.6, exact=exact))
    t, i = C.shock_faces()
    vals = np.zeros((6, 5))
    vals[0] = inlet
    b = s.add_block(*SHAPE, t, i, vals)
    s.set_nodes(b, *nodes)
    s.finalize()
    s.set_q(b, q0)
    dts = []
    for _ in range(STEPS):
        s.step(1)
        dts.append(s.time_dt()[1])
    out = s.get_q(b), np.array(dts), s.time_dt()[0], s.residual()
    s.close()
    return out


@pytest.mark.gpu
def test_shock_turbulence_bitwise(ref):
    q, dts, t, res = _gpu(exact=True)
    qr, dtr, tr, resr = ref
    assert np.array_equal(dts, dtr) and t == tr[-1]
    assert np.array_equal(q, qr), float(np.max(np.abs(q - qr)) / np.max(np.abs(qr)))
    assert res == resr[-1]


@pytest.mark.gpu
def test_shock_turbulence_fast(ref):
    q, dts, _, _ = _gpu(exact=False)
    qr = ref[0]
    assert float(np.max(np.abs(q - qr)) / np.max(np.abs(qr))) < 1e-11
