"""100 TVD-RK3 steps of the 64^3 Navier-Stokes Taylor-Green case (WENO5-JS, LF, cd6,
CFL 0.5, Re 1600, Ma 0.1) against the reference itself.

The reference runs here as 8 MPI ranks (2x2x2 blocks of 32^3, the project's shared-memory
MPI shim); its multi-rank result equals its single-block result bit for bit for explicit
WENO schemes.  The GPU runs the single 64^3 block.  Criterion for the reference-order build:
bitwise equal.

The throughput build cannot be held to a fixed tolerance at CFL 0.5: this discretisation
amplifies the (pi, pi, pi) checkerboard mode of the grid by about 4.6x per step, so a
1e-15 relative perturbation of the initial state alone, stepped in the reference's own
arithmetic, ends 100 steps at a few 1e-2 relative difference (the mode saturates).  Its
criteria are therefore (a) no further from the reference than that perturbed reference-order
run, (b) conserved totals of the periodic box unchanged to round-off, and (c) at CFL 0.2,
where the mode is damped and perturbations stay at round-off, within 1e-12 of the
reference-order build after the same 100 steps.
"""
import math

import numpy as np
import pytest

from oracle import refrun as R

N = 64
STEPS = 100
PARAMS = {"Reynolds": 1600.0, "Mach": 0.1, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
          "T_inf": 288.0, "T_wall": 1.0}


def _reference():
    x, y, z = R.box_nodes(N, N, N, hi=(2.0 * math.pi,) * 3)
    one = R.Case(model="NavierStokes3d", riemann="LF", schemes=("weno5js",) * 3, params=PARAMS,
                 benchmark=2, nodes=[(x, y, z)], bc_topo=[R.PERIODIC_SELF])
    q0 = R.stack(R.run(one, "init")[0], "Q", 5)
    h = N // 2
    nodes, topo = [], []
    rank = lambda a, b, c: a + 2 * (b + 2 * c)  # noqa: E731
    for c in range(2):
        for b in range(2):
            for a in range(2):
                sl = (slice(c * h, c * h + h + 1), slice(b * h, b * h + h + 1), slice(a * h, a * h + h + 1))
                nodes.append((x[sl], y[sl], z[sl]))
                pos = [a, b, c]
                lines = []
                for f in range(6):
                    d, side = f // 2, f % 2
                    p2 = list(pos)
                    p2[d] = (p2[d] + (1 if side else -1)) % 2
                    lines.append(f"{rank(*p2)} {f ^ 1}")
                topo.append(lines)
    multi = R.Case(model="NavierStokes3d", riemann="LF", schemes=("weno5js",) * 3, params=PARAMS,
                   benchmark=2, nodes=nodes, bc_topo=topo)
    out = R.run(multi, "steps", STEPS, timeout=1800)
    q = np.zeros((5, N, N, N))
    for r, d in enumerate(out):
        a, b, c = r % 2, (r // 2) % 2, r // 4
        q[:, c * h:(c + 1) * h, b * h:(b + 1) * h, a * h:(a + 1) * h] = R.stack(d, "Q", 5)
    return (x, y, z), q0, q, out[0]["dt"], out[0]["time"]


@pytest.fixture(scope="module")
def reference():
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    return _reference()


def _gpu(nodes, q0, exact, cfl=0.5):
    import nuc3d_b200 as nb
    cfg = nb.Config(scheme_ivs=("weno5js",) * 3, riemann="LF", model="NavierStokes3d",
                    reynolds=1600.0, mach=0.1, prandtl=0.72, exact=exact, cfl=cfl)
    s = nb.Solver(cfg)
    b = s.add_block(N, N, N, [0] * 6, [1, 0, 3, 2, 5, 4])
    s.set_mesh(b, *nodes)
    s.finalize()
    s.set_q(b, q0)
    s.step(STEPS)
    t, dt = s.time_dt()
    return s.get_q(b), t, dt


@pytest.mark.gpu
@pytest.mark.slow
def test_tgv64_100_steps_bitwise(reference):
    nodes, q0, qref, dts, times = reference
    q, t, dt = _gpu(nodes, q0, exact=True)
    assert t == times[-1] and dt == dts[-1]
    assert np.array_equal(q, qref), float(np.max(np.abs(q - qref)) / np.max(np.abs(qref)))


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
@pytest.mark.slow
def test_tgv64_100_steps_fast_within_input_sensitivity(reference):
    nodes, q0, qref, dts, times = reference
    q, t, dt = _gpu(nodes, q0, exact=False)
    rng = np.random.default_rng(20261203)
    q0p = q0 * (1.0 + 1e-15 * rng.standard_normal(q0.shape))
    qp, _, _ = _gpu(nodes, q0p, exact=True)
    rel_fast, rel_pert = _rel(q, qref), _rel(qp, qref)
    assert rel_pert > 1e-6, rel_pert          # the checkerboard mode did grow
    assert rel_fast <= 4.0 * rel_pert, (rel_fast, rel_pert)
    assert abs(t - times[-1]) <= 1e-6 * times[-1], (t, times[-1])
    # conserved totals of the periodic box (mass, momentum, energy); momentum components
    # against the total momentum magnitude (w starts at exactly zero)
    for v in range(5):
        s0, s1 = q0[v].sum(), q[v].sum()
        scale = np.abs(q0[1:4]).sum() if 1 <= v <= 3 else np.abs(q0[v]).sum()
        assert abs(s1 - s0) <= 1e-12 * scale, (v, s0, s1)


@pytest.mark.gpu
@pytest.mark.slow
def test_tgv64_100_steps_fast_stable_cfl(reference):
    nodes, q0, _, _, _ = reference
    qe, te, _ = _gpu(nodes, q0, exact=True, cfl=0.2)
    qf, tf, _ = _gpu(nodes, q0, exact=False, cfl=0.2)
    assert _rel(qf, qe) <= 1e-12, _rel(qf, qe)
    assert abs(tf - te) <= 1e-13 * te
