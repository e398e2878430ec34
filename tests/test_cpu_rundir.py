"""The run-directory reader and the restart files (nuc3d_b200/rundir.py), on the host: the
reference's input files parsed with its defaults and fallbacks (src/fieldOperator.cpp,
src/physicsModel.cpp, src/IOcontroller.cpp), its refusals raised as errors, and the
restart format (a little-endian double time, then the five components) round-tripped."""
import math
import struct

import numpy as np
import pytest

from nuc3d_b200 import rundir as RD


def _write(root, rel, text):
    p = root / rel
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(text)
    return p


def test_method_defaults_and_fallbacks(tmp_path):
    _write(tmp_path, "inp/Method.in", "scheme_x_ivs weno5z\nscheme_y_ivs nosuch\nscheme_z_vis cd8\n"
                                      "scheme_y_vis nosuch\n")
    m = RD.read_method(tmp_path)
    assert m["scheme_x_ivs"] == "weno5z"
    assert m["scheme_y_ivs"] == "weno5js"  # unknown name: the reference's weno5js
    assert m["scheme_z_ivs"] == "weno5js"  # absent: the default
    assert m["scheme_z_vis"] == "cd8" and m["scheme_y_vis"] == "cd6" and m["scheme_x_vis"] == "cd6"


def test_physmodel_positional_and_parameters(tmp_path):
    _write(tmp_path, "inp/PhysModel.in",
           "neqs 5\neos_type Ideal\nriemann_type AUSM\nmodel NavierStokes3d\nvis_type Sutherland\n"
           "Reynolds 1600\nMach 0.1\n")
    p = RD.read_phys(tmp_path)
    assert (p["neqs"], p["riemann"], p["model"]) == (5, "AUSM", "NavierStokes3d")
    assert p["params"]["Reynolds"] == 1600.0 and p["params"]["Mach"] == 0.1
    assert p["params"]["Gamma"] == 1.4 and p["params"]["T_wall"] == 1.0  # defaults


def test_physmodel_refusals(tmp_path):
    base = "neqs 5\neos_type Ideal\nriemann_type {r}\nmodel Euler3d\nvis_type Sutherland\n"
    _write(tmp_path, "inp/PhysModel.in", base.format(r="Roe"))
    with pytest.raises(ValueError, match="Riemann"):
        RD.read_phys(tmp_path)
    _write(tmp_path, "inp/PhysModel.in", base.format(r="LF") + "Prandtl 0.7\n")
    with pytest.raises(ValueError, match="unknown parameter"):
        RD.read_phys(tmp_path)


def test_iocontroller_types(tmp_path):
    _write(tmp_path, "inp/IOController.in", "startStep 0\nendStep 40\nsaveStep 10\ncfl 0.3\n"
                                            "tl 1.5\nBinary no\nBenchmark 2\n")
    io = RD.read_io(tmp_path)
    assert io["endStep"] == 40 and isinstance(io["endStep"], int)
    assert io["cfl"] == 0.3 and io["tl"] == 1.5 and io["Binary"] == "no" and io["Benchmark"] == 2
    assert io["postStep"] == 1  # default


def test_postproc_required(tmp_path):
    with pytest.raises(ValueError, match="PostProc"):
        RD.read_postproc(tmp_path)
    _write(tmp_path, "inp/PostProc.in", "a 1\nb 0\nSimutaneousData 1\nd 0\ne 5\n")
    assert RD.read_postproc(tmp_path) == [1, 0, 1, 0, 5]


def test_mesh_and_truncation(tmp_path):
    n = (3, 2, 2)  # nodes
    x = np.arange(12, dtype=float) * 0.5
    body = " ".join(f"{v:.17g}" for v in np.concatenate([x, x + 1.0, x + 2.0]))
    p = _write(tmp_path, "mesh/mesh_0.x", f"{n[0]} {n[1]} {n[2]}\n{body}\n")
    X, Y, Z = RD.read_mesh(p)
    assert X.shape == (2, 2, 3) and X[0, 0, 1] == 0.5 and Z[1, 1, 2] == x[11] + 2.0
    p.write_text(f"{n[0]} {n[1]} {n[2]}\n" + " ".join(body.split()[:-1]))
    with pytest.raises(ValueError, match="end of file"):
        RD.read_mesh(p)


def test_bc_topo(tmp_path):
    p = _write(tmp_path, "bc_topo/BC_Topo_0.in",
               "-1 0 1.0 0.5 0 0 0.7\n-1 1\n3 2\n1 3\n0 5\n0 4\n")
    t, i, v = RD.read_bc_topo(p)
    assert t == [-1, -1, 3, 1, 0, 0] and i == [0, 1, 2, 3, 5, 4]
    assert list(v[0]) == [1.0, 0.5, 0.0, 0.0, 0.7] and not v[1:].any()
    p.write_text("-1 0\n-1 1\n")
    with pytest.raises(ValueError, match="fewer than 6"):
        RD.read_bc_topo(p)


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    q = rng.standard_normal((5, 4, 3, 2))
    path = RD.restart_path(tmp_path, 20, 1)
    assert path.name == "NUC3d_step_20_ID_1.bin" and path.parent.name == "flowData"
    RD.write_restart(path, 0.125, q)
    raw = path.read_bytes()
    assert len(raw) == 8 + q.size * 8 and struct.unpack("<d", raw[:8])[0] == 0.125
    t, q2 = RD.read_restart(path, (4, 3, 2))
    assert t == 0.125 and np.array_equal(q2, q)


def test_initial_q_taylor_green_and_default():
    shape = (4, 4, 4)
    h = 2.0 * math.pi / 4
    c = (np.arange(4) + 0.5) * h
    Z, Y, X = np.meshgrid(c, c, c, indexing="ij")
    jac = np.full(shape, 2.0)
    g, ma = 1.4, 0.1
    q = RD.initial_q(2, (X, Y, Z), jac, g, ma)
    rho = q[0] * jac
    u = q[1] * jac / rho
    assert np.allclose(rho, 1.0) and np.allclose(u, np.sin(X) * np.cos(Y) * np.cos(Z), atol=1e-15)
    p = (g - 1.0) * (q[4] * jac - 0.5 * rho * ((q[1] * jac) ** 2 + (q[2] * jac) ** 2) / rho ** 2)
    p_ref = 1.0 / (g * ma * ma) + ((np.cos(2 * Z) + 2.0) * (np.cos(2 * X) + np.cos(2 * Y)) - 2.0) / 16.0
    assert np.allclose(p, p_ref, rtol=1e-12)
    q0 = RD.initial_q(0, (X, Y, Z), jac, g, 0.5)
    assert np.allclose(q0[1] * jac, 1.0) and np.allclose(q0[2:4], 0.0)
