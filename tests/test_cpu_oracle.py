"""The C restatement (oracle/nuc3d_oracle.c) reproduces the reference's golden vectors
bit for bit: metrics, one right-hand side, dt, and the state after 1 and n steps."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G


def oracle_run(g):
    r = O.Run(g.cfg["schemes"], g.cfg["riemann"], g.cfg["model"], g.cfg["params"])
    t, i, v = G.bc_arrays(g)
    r.add_block(O.metrics(*G.nodes(g)), t, i, v, g.q0)
    return r


def test_oracle_metrics_bitwise():
    g = G.load("tgv_ns_weno5js_lf")
    m = O.metrics(*G.nodes(g))
    assert np.array_equal(m["jac"], g.metrics_jac)
    for nm in ("xi_xyz", "eta_xyz", "zeta_xyz", "dxyz"):
        assert np.array_equal(m[nm], g.data[f"metrics_{nm}"]), nm


@pytest.mark.parametrize("name", G.names())
def test_oracle_rhs_bitwise(name):
    g = G.load(name)
    dt, rhs = oracle_run(g).rhs()
    assert dt == g.dt_local[0]
    assert np.array_equal(rhs[0], g.rhs), np.max(np.abs(rhs[0] - g.rhs))


@pytest.mark.parametrize("name", G.names())
def test_oracle_steps_bitwise(name):
    g = G.load(name)
    r = oracle_run(g)
    dt, t = r.step(1)
    assert np.array_equal(r.q(0), g.q1)
    assert dt[0] == g.dt[0]
    n = int(g.cfg["nsteps"])
    r = oracle_run(g)
    dt, t = r.step(n)
    assert np.array_equal(r.q(0), g.qn), np.max(np.abs(r.q(0) - g.qn))
    assert np.array_equal(dt, g.dt) and t == g.time[-1]
