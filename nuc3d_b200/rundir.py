"""Run a NUC3d run directory on the GPU: the reference's input files in, its restart files out.

    python -m nuc3d_b200.run RUNDIR [--steps N] [--fast]

Reads, relative to RUNDIR, what the reference's singleBlock reads
(src/singleBlock.cpp:10-43, src/block.cpp:31-100):
  inp/Method.in        scheme_{x,y,z}_ivs / _vis (src/fieldOperator.cpp:20-87)
  inp/PhysModel.in     5 positional lines, then Reynolds Mach Pt Gamma T_ref T_inf T_wall
                       (src/physicsModel.cpp:59-102)
  inp/IOController.in  startStep endStep saveStep Benchmark cfl tl Binary ...
                       (src/IOcontroller.cpp:12-64, ifsolve/ifsave :181-203)
  mesh/mesh_<r>.x      one file per rank = one block here (src/block.cpp:42-81)
  bc_topo/BC_Topo_<r>.in   faces xi-,xi+,eta-,eta+,zeta-,zeta+ (src/boundaryConditions.cpp:25-93);
                       a neighbour rank r becomes block r of one GPU context
  flowData/NUC3d_step_<s>_ID_<r>.bin  restart state when startStep > 0 (src/block.cpp:785-855)
  inp/PostProc.in      5 positional ints; SimutaneousData (the third) 1 asks for
                       postproc::solveQ (src/postproc.cpp:29-67, 247-260)
and writes flowData/NUC3d_step_<s>_ID_<r>.bin every saveStep steps when Binary is "yes"
(src/block.cpp:754-783) and, every postStep steps when SimutaneousData is 1, appends
"step time enstrophy kinetic" to enstrophy.dat (src/postproc.cpp:836-846), with the
loop of singleBlock::solvePDE (src/singleBlock.cpp:51-71): step while time <= tl and
step < endStep; post-process, then save.
Initial states for startStep == 0 follow block::initialQ (src/block.cpp:523-567) with the
Benchmark initialisers default / isentropic vortex / Taylor-Green (:658-690), evaluated with
the C library's sin/cos/exp/pow through Python's math module.
"""
from __future__ import annotations

import argparse
import math
import struct
import sys
import time as _time
from pathlib import Path

import numpy as np

from . import Config, Solver
from .metrics import metrics_from_nodes

METHOD_DEFAULTS = {"scheme_time": "RK3", "scheme_x_ivs": "weno5js", "scheme_y_ivs": "weno5js",
                   "scheme_z_ivs": "weno5js", "scheme_x_vis": "cd6", "scheme_y_vis": "cd6",
                   "scheme_z_vis": "cd6"}
PHYS_DEFAULTS = {"Reynolds": 1000.0, "Mach": 0.5, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
                 "T_inf": 288.0, "T_wall": 1.0}
IO_INT = {"startStep": 0, "endStep": 100000, "saveStep": 1000, "postStep": 1, "Benchmark": 0}
IO_DBL = {"cfl": 0.5, "tl": 0.0, "dt": 0.01}
IO_STR = {"Binary": "yes", "Tecplot": "yes", "PostProc": "yes"}
KNOWN_SCHEMES = ("weno5js", "weno5z", "weno7js", "crweno5", "hccs", "hccs77", "weno3js", "upwind1st")
KNOWN_VIS = ("cd2", "cd6", "cd8")


def _pairs(path: Path):
    words = path.read_text().split()
    return [(words[i], words[i + 1]) for i in range(0, len(words) - 1, 2)]


def read_method(rundir: Path) -> dict:
    m = dict(METHOD_DEFAULTS)
    for k, v in _pairs(rundir / "inp/Method.in"):
        if k in m:
            m[k] = v
    for ax in "xyz":
        if m[f"scheme_{ax}_ivs"] not in KNOWN_SCHEMES:
            # the reference falls back to weno5js for unknown names (src/fieldOperator.cpp:171-174)
            m[f"scheme_{ax}_ivs"] = "weno5js"
        if m[f"scheme_{ax}_vis"] not in KNOWN_VIS:
            # and to cd6 for unknown viscous schemes (src/fieldOperator.cpp:298-301)
            m[f"scheme_{ax}_vis"] = "cd6"
    return m


def read_phys(rundir: Path) -> dict:
    words = (rundir / "inp/PhysModel.in").read_text().split()
    # the first five entries are positional "name value" pairs (src/physicsModel.cpp:65-69)
    pos = [words[2 * i + 1] for i in range(5)]
    p = {"neqs": int(pos[0]), "eos": pos[1], "riemann": pos[2], "model": pos[3], "vis": pos[4]}
    params = dict(PHYS_DEFAULTS)
    rest = words[10:]
    for i in range(0, len(rest) - 1, 2):
        if rest[i] not in params:
            raise ValueError(f"PhysModel.in: unknown parameter {rest[i]} (the reference exits)")
        params[rest[i]] = float(rest[i + 1])
    if p["riemann"] not in ("LF", "AUSM", "AUSMp"):
        raise ValueError(f"PhysModel.in: Riemann solver {p['riemann']} does not exist")
    p["params"] = params
    return p


def read_io(rundir: Path) -> dict:
    io = {**IO_INT, **IO_DBL, **IO_STR}
    for k, v in _pairs(rundir / "inp/IOController.in"):
        if k in IO_INT:
            io[k] = int(v)
        elif k in IO_DBL:
            io[k] = float(v)
        elif k in IO_STR:
            io[k] = v
    return io


def read_postproc(rundir: Path) -> list[int]:
    """The positional integers of inp/PostProc.in (the reference exits without the file)."""
    path = rundir / "inp/PostProc.in"
    if not path.exists():
        raise ValueError("inp/PostProc.in does not exist (the reference exits)")
    words = path.read_text().split()
    return [int(words[i + 1]) for i in range(0, len(words) - 1, 2)]


def read_mesh(path: Path):
    toks = path.read_text().split()
    nx0, ny0, nz0 = (int(t) for t in toks[:3])
    n = nx0 * ny0 * nz0
    vals = np.array(toks[3:3 + 3 * n], dtype=np.float64)
    if vals.size != 3 * n:
        raise ValueError(f"{path}: end of file (the reference exits)")
    return [vals[k * n:(k + 1) * n].reshape(nz0, ny0, nx0) for k in range(3)]


def read_bc_topo(path: Path):
    types, ids, vals = [], [], np.zeros((6, 5))
    lines = [ln for ln in path.read_text().splitlines()][:6]
    if len(lines) < 6:
        raise ValueError(f"{path}: fewer than 6 faces")
    for f, ln in enumerate(lines):
        w = ln.split()
        types.append(int(w[0]))
        ids.append(int(w[1]))
        extra = [float(x) for x in w[2:7]]
        vals[f, :len(extra)] = extra
    return types, ids, vals


def restart_path(rundir: Path, step: int, rank: int) -> Path:
    return rundir / f"flowData/NUC3d_step_{step}_ID_{rank}.bin"


def read_restart(path: Path, shape):
    raw = path.read_bytes()
    t = struct.unpack("<d", raw[:8])[0]
    q = np.frombuffer(raw[8:], dtype="<f8").reshape((5,) + shape)
    return t, q.copy()


def write_restart(path: Path, t: float, q: np.ndarray) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as f:
        f.write(struct.pack("<d", t))
        f.write(np.ascontiguousarray(q, dtype="<f8").tobytes())


def initial_q(bench: int, centre, jac, gamma, mach):
    """block::initialQ with the Benchmark initialisers (src/block.cpp:523-567,658-690)."""
    sin, cos, exp = (np.frompyfunc(f, 1, 1) for f in (math.sin, math.cos, math.exp))
    x, y, z = centre
    if bench == 2:
        u = (sin(x) * cos(y) * cos(z)).astype(np.float64)
        v = (-cos(x) * sin(y) * cos(z)).astype(np.float64)
        w = np.zeros_like(u)
        rho = np.ones_like(u)
        p = 1.0 / (gamma * mach * mach) + ((cos(2.0 * z).astype(np.float64) + 2.0) *
                                           (cos(2.0 * x).astype(np.float64) +
                                            cos(2.0 * y).astype(np.float64)) - 2.0) / 16.0
    elif bench == 1:
        pie = 4.0 * math.atan(1.0)
        b, xc, yc = 0.5, 5.0, 5.0
        r = np.sqrt((x - xc) * (x - xc) + (y - yc) * (y - yc))
        pw = np.frompyfunc(math.pow, 2, 1)
        rho = pw(1 - (gamma - 1.0) * b * b * exp(1 - r * r).astype(np.float64) / (8.0 * gamma * pie * pie),
                 2.5).astype(np.float64)
        e2 = exp((1 - r * r) / 2).astype(np.float64)
        u = 0.5 - b / (2.0 * pie) * e2 * (y - yc)
        v = b / (2.0 * pie) * e2 * (x - xc)
        w = np.zeros_like(u)
        p = pw(rho, gamma).astype(np.float64)
    else:
        rho = np.ones_like(x)
        u = np.ones_like(x)
        v = np.zeros_like(x)
        w = np.zeros_like(x)
        p = np.full_like(x, 1.0 / (mach * mach * gamma))
    rhoe = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho / jac, (rho * u) / jac, (rho * v) / jac, (rho * w) / jac, rhoe / jac])


def run(rundir, steps: int | None = None, exact: bool = True, quiet: bool = False) -> dict:
    rundir = Path(rundir)
    method = read_method(rundir)
    phys = read_phys(rundir)
    io = read_io(rundir)
    post = read_postproc(rundir)
    solve_q = len(post) > 2 and post[2] == 1
    if len(post) > 2 and post[2] not in (0, 1):
        raise ValueError(f"PostProc.in: no such postproc for {post[2]} (the reference exits)")
    prm = phys["params"]
    cfg = Config(scheme_ivs=tuple(method[f"scheme_{a}_ivs"] for a in "xyz"),
                 scheme_vis=tuple(method[f"scheme_{a}_vis"] for a in "xyz"),
                 riemann=phys["riemann"], model=phys["model"], reynolds=prm["Reynolds"],
                 mach=prm["Mach"], prandtl=prm["Pt"], gamma=prm["Gamma"], t_ref=prm["T_ref"],
                 t_inf=prm["T_inf"], t_wall=prm["T_wall"], cfl=io["cfl"], exact=exact)
    meshes = sorted(rundir.glob("mesh/mesh_*.x"), key=lambda p: int(p.stem.split("_")[1]))
    s = Solver(cfg)
    shapes, metrics = [], []
    start = io["startStep"]
    for r, mp in enumerate(meshes):
        x, y, z = read_mesh(mp)
        t, i, v = read_bc_topo(rundir / f"bc_topo/BC_Topo_{r}.in")
        nz, ny, nx = (d - 1 for d in x.shape)
        b = s.add_block(nx, ny, nz, t, i, v)
        symm = any(tt == -1 and ii == 3 for tt, ii in zip(t, i))
        if start > 0 and not symm:
            s.set_nodes(b, x, y, z)           # metrics on the GPU
            metrics.append(None)
        else:                                  # cell centres (initial state) or dxyz needed
            metrics.append(s.set_mesh(b, x, y, z))
        shapes.append((nz, ny, nx))
    s.finalize()
    t0 = 0.0
    for r, sh in enumerate(shapes):
        if start > 0:
            t0, q = read_restart(restart_path(rundir, start, r), sh)
        else:
            m = metrics[r]
            q = initial_q(io["Benchmark"], m["xyz_center"], m["jac"], prm["Gamma"], prm["Mach"])
        s.set_q(r, q)
    s.set_time(t0)
    step, t = start, t0
    end = io["endStep"] if steps is None else start + steps
    while t <= io["tl"] and step < end:
        w0 = _time.perf_counter()
        s.step(1)
        t, dt = s.time_dt()
        step += 1
        if not quiet:
            print(f"========step = {step}\n time = {t:.6g}, dt = {dt:.6g}, "
                  f"GPU time = {_time.perf_counter() - w0:.6g}(s) ", flush=True)
        if solve_q and io["postStep"] != 0 and step % io["postStep"] == 0:
            ens, kin = s.diagnostics()
            with open(rundir / "enstrophy.dat", "a") as f:
                f.write(f"{step} {t:.12g} {ens:.12g} {kin:.12g}\n")
        if io["Binary"] == "yes" and step % io["saveStep"] == 0:
            for r in range(len(shapes)):
                write_restart(restart_path(rundir, step, r), t, s.get_q(r))
    out = {"step": step, "time": t, "q": [s.get_q(r) for r in range(len(shapes))]}
    s.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("rundir")
    ap.add_argument("--steps", type=int, default=None, help="override endStep - startStep")
    ap.add_argument("--fast", action="store_true", help="throughput arithmetic (default: reference order)")
    a = ap.parse_args(argv)
    run(a.rundir, a.steps, exact=not a.fast)
    return 0


if __name__ == "__main__":
    sys.exit(main())
