"""The step's residual and the stage-by-stage entry points against the reference.

block::solve prints a residual every step (PDEData3d::setRES, src/PDEData3d.cpp:90-122);
the golden fixtures hold the reference's value after each of their steps.  A host that
drives the reference's own loop (EulerData3D::solve, then PDEData3d::solve ->
tvdrk3rd::integrationAll) calls nuc3d_rhs_stage and nuc3d_rk_stage per stage; three such
pairs are one nuc3d_step."""
import numpy as np
import pytest

from tests import golden_cases as G

CASES = ["tgv_ns_weno5js_lf", "sphere_euler_weno5z_ausm_outlet", "sphere_reset_euler_weno5z_ausm",
         "bc_ns_weno7js_ausmp", "crweno5_euler_lf_periodic", "mixed_low_order_ausmp"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_residual_every_step(name):
    g = G.load(name)
    s = G.solver(g, exact=True)
    f = G.solver(g, exact=False)
    for k in range(int(g.cfg["nsteps"])):
        s.step(1)
        f.step(1)
        assert s.residual() == g.res[k], (k, s.residual(), g.res[k])
        assert abs(f.residual() - g.res[k]) <= 1e-9 * abs(g.res[k]), (k, f.residual(), g.res[k])


@pytest.mark.gpu
def test_residual_two_ranks_is_the_maximum():
    name = G.multi_names()[0]
    mr = G.load_multi(name)
    g = G.load(name)
    from tests.test_gpu_parity import _two_rank_solver
    s, _ = _two_rank_solver(g, exact=True)
    s.step(int(mr["nsteps"][0]))
    assert s.residual() == mr["res"][-1]


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("exact", [True, False])
def test_stage_by_stage_equals_step(name, exact):
    """rhs_stage(s) + rk_stage(s, dt) for s = 0, 1, 2 with dt = cfl * dt_local of stage 0,
    as PDEData3d::solve fixes it (src/PDEData3d.cpp:74-80), is nuc3d_step: the state, time,
    dt and residual; the reference-order build also equals the reference's step.  The
    throughput build's residual sums per cell tile here and per sweep tile in the step, so
    it agrees to round-off."""
    g = G.load(name)
    a = G.solver(g, exact=exact)
    b = G.solver(g, exact=exact)
    for k in range(2):
        dt = 0.0
        for st in range(3):
            dl = a.rhs_stage(st)
            if st == 0:
                dt = 0.5 * dl
            a.rk_stage(st, dt)
        a.sync()
        b.step(1)
        assert np.array_equal(a.get_q(0), b.get_q(0)), k
        assert a.time_dt() == b.time_dt()
        if exact:
            assert a.residual() == b.residual()
        else:
            assert abs(a.residual() - b.residual()) <= 1e-12 * b.residual()
        if exact and k == 0:
            assert np.array_equal(a.get_q(0), g.q1)
            assert a.residual() == g.res[0]
