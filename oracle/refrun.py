"""Run the NUC3d reference (built under oracle/_ref) on a generated case.

TEST INFRASTRUCTURE ONLY: used by tests/, tests/golden/make_golden.py and the
CPU-baseline leg of bench.py.  Nothing in the GPU product imports it.

The reference reads a run directory laid out as (paths relative to its cwd):

  inp/Method.in        key value   (src/fieldOperator.cpp:20-33)
  inp/PhysModel.in     5 positional lines, then key value (src/physicsModel.cpp:59-102)
  inp/IOController.in  key value   (src/IOcontroller.cpp:12-64)
  inp/PostProc.in      5 positional ints (src/postproc.cpp:29-67)
  mesh/mesh_<r>.x      node dims, then x, y, z node fields, i fastest (src/block.cpp:42-81)
  bc_topo/BC_Topo_<r>.in  6 lines "type id [values]", faces xi-,xi+,eta-,eta+,zeta-,zeta+
                       (src/boundaryConditions.cpp:25-93)
  flowData/NUC3d_step_<s>_ID_<r>.bin  restart: f64 time, then 5 fields of Q=U/J
                       (src/block.cpp:785-855), read when startStep > 0

This module writes such a directory, runs oracle/_ref/nuc3d_ref_taps in it and
parses the "NUCT" dumps that harness writes (see oracle/ref_taps.cpp).
"""
from __future__ import annotations

import os
import shutil
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_BIN_DIR = ORACLE_DIR / "_ref"


def ref_binary(name: str = "nuc3d_ref_taps") -> Path:
    p = REF_BIN_DIR / name
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `make -C oracle ref` (needs the reference sources)")
    return p


@dataclass
class Case:
    """One single-rank or multi-rank run of the reference."""

    model: str = "Euler3d"              # Euler3d | NavierStokes3d
    riemann: str = "LF"                 # LF | AUSM | AUSMp
    schemes: tuple = ("weno5js", "weno5js", "weno5js")
    vis: tuple = ("cd6", "cd6", "cd6")
    params: dict = field(default_factory=lambda: {
        "Reynolds": 1600.0, "Mach": 0.1, "Pt": 0.72, "Gamma": 1.4,
        "T_ref": 110.4, "T_inf": 288.0, "T_wall": 1.0})
    cfl: float = 0.5
    benchmark: int = 0                  # initialiser index when startStep == 0
    start_step: int = 0                 # > 0: Q comes from the restart file
    post_q: bool = False                # PostProc.in SimutaneousData 1 (postproc::solveQ)
    # per rank: node coordinates x, y, z each shaped (nz+1, ny+1, nx+1)
    nodes: list = field(default_factory=list)
    # per rank: 6 strings "type id [values...]"
    bc_topo: list = field(default_factory=list)
    # per rank (only if start_step > 0): Q = U/J shaped (5, nz, ny, nx)
    q0: list = field(default_factory=list)
    time0: float = 0.0

    @property
    def nranks(self) -> int:
        return len(self.nodes)


def _fmt(x: float) -> str:
    return repr(float(x))


def write_case(case: Case, rundir: Path) -> None:
    rundir = Path(rundir)
    for d in ("inp", "mesh", "bc_topo", "flowData"):
        (rundir / d).mkdir(parents=True, exist_ok=True)
    sx, sy, sz = case.schemes
    vx, vy, vz = case.vis
    (rundir / "inp/Method.in").write_text(
        f"scheme_time RK3\nscheme_x_ivs {sx}\nscheme_y_ivs {sy}\nscheme_z_ivs {sz}\n"
        f"scheme_x_vis {vx}\nscheme_y_vis {vy}\nscheme_z_vis {vz}\n")
    lines = ["neqs 5", "EoS IdealGas", f"Riemann {case.riemann}", f"Model {case.model}",
             "Vis Sutherland"]
    for k in ("Reynolds", "Mach", "Pt", "Gamma", "T_ref", "T_inf", "T_wall"):
        lines.append(f"{k} {_fmt(case.params[k])}")
    (rundir / "inp/PhysModel.in").write_text("\n".join(lines) + "\n")
    (rundir / "inp/IOController.in").write_text(
        f"startStep {case.start_step}\nendStep 1000000000\nsaveStep 1000000000\npostStep 0\n"
        f"Benchmark {case.benchmark}\ncfl {_fmt(case.cfl)}\ntl 1e300\ndt 0.01\n"
        "Binary no\nTecplot no\nPostProc no\n")
    (rundir / "inp/PostProc.in").write_text(
        f"AverageType 0\nAverageStartStep 0\nSimutaneousData {int(case.post_q)}\nAveragedSaveType 0\n"
        "SimutaneousSaveType 0\n")
    for r, xyz in enumerate(case.nodes):
        x, y, z = (np.asarray(a, dtype=np.float64) for a in xyz)
        nz0, ny0, nx0 = x.shape
        with open(rundir / f"mesh/mesh_{r}.x", "w") as f:
            f.write(f"{nx0} {ny0} {nz0}\n")
        with open(rundir / f"mesh/mesh_{r}.x", "a") as f:
            for a in (x, y, z):
                # %.17g round-trips every double exactly
                np.ascontiguousarray(a).ravel().tofile(f, sep="\n", format="%.17g")
                f.write("\n")
        (rundir / f"bc_topo/BC_Topo_{r}.in").write_text("\n".join(case.bc_topo[r]) + "\n")
        if case.start_step > 0:
            q = np.ascontiguousarray(case.q0[r], dtype=np.float64)
            with open(rundir / f"flowData/NUC3d_step_{case.start_step}_ID_{r}.bin", "wb") as f:
                f.write(struct.pack("<d", case.time0))
                f.write(q.tobytes())


def read_nuct(path: Path) -> dict:
    out = {}
    with open(path, "rb") as f:
        if f.read(4) != b"NUCT":
            raise ValueError(f"{path}: not a NUCT dump")
        while True:
            h = f.read(4)
            if not h:
                break
            (nl,) = struct.unpack("<I", h)
            name = f.read(nl).decode()
            (nd,) = struct.unpack("<I", f.read(4))
            dims = struct.unpack(f"<{nd}q", f.read(8 * nd))
            n = int(np.prod(dims))
            out[name] = np.frombuffer(f.read(8 * n), dtype="<f8").reshape(dims).copy()
    return out


def stack(d: dict, name: str, n: int) -> np.ndarray:
    return np.stack([d[f"{name}.{i}"] for i in range(n)])


def run(case: Case, mode: str, *args, binary: str = "nuc3d_ref_taps", keep: Path | None = None,
        timeout: float = 3600.0, stdout: list | None = None) -> list:
    """Run the taps harness; returns one dict of arrays per rank.  stdout (a list), if
    given, receives the reference's standard output (all ranks)."""
    tmp = Path(keep) if keep else Path(tempfile.mkdtemp(prefix="nuc3d_ref_"))
    try:
        write_case(case, tmp)
        env = dict(os.environ, NUC_SHIM_NP=str(case.nranks))
        out = tmp / "dump.nuct"
        argv = [str(ref_binary(binary)), mode, *[str(a) for a in args]]
        if mode in ("init", "rhs", "steps", "post"):
            argv.append(str(out))
        p = subprocess.run(argv, cwd=tmp, env=env, capture_output=True, text=True,
                           timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference failed ({p.returncode}):\n{p.stdout[-2000:]}\n"
                               f"{p.stderr[-2000:]}")
        if stdout is not None:
            stdout.append(p.stdout)
        if mode == "time":
            return [p.stdout]
        return [read_nuct(Path(f"{out}.r{r}")) for r in range(case.nranks)]
    finally:
        if keep is None:
            shutil.rmtree(tmp, ignore_errors=True)


# ----------------------------------------------------------------------------------
# Case builders used by the fixtures, the tests and the CPU baseline.
# Node coordinates use only + - * / so every IEEE machine produces the same bits.
# ----------------------------------------------------------------------------------

def box_nodes(nx, ny, nz, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), wavy=0.0):
    """(x, y, z) node arrays of a box, optionally with a smooth polynomial distortion."""
    i = np.arange(nx + 1, dtype=np.float64) / nx
    j = np.arange(ny + 1, dtype=np.float64) / ny
    k = np.arange(nz + 1, dtype=np.float64) / nz
    K, J, I = np.meshgrid(k, j, i, indexing="ij")
    if wavy:
        bi = I * (1.0 - I)
        bj = J * (1.0 - J)
        bk = K * (1.0 - K)
        I = I + wavy * bi * (0.5 - J) * (1.0 + K)
        J = J + wavy * bj * (I - 0.5) * (1.0 - 0.5 * K)
        K = K + wavy * bk * (0.5 - I) * J
    x = lo[0] + (hi[0] - lo[0]) * I
    y = lo[1] + (hi[1] - lo[1]) * J
    z = lo[2] + (hi[2] - lo[2]) * K
    return x, y, z


PERIODIC_SELF = ["0 1", "0 0", "0 3", "0 2", "0 5", "0 4"]


def bc_lines(kinds, values=None):
    """kinds: 6 of 'periodic' | 'inlet' | 'outlet' | 'wall' | 'symm' (single block)."""
    ids = {"inlet": 0, "outlet": 1, "wall": 2, "symm": 3}
    out = []
    for f, k in enumerate(kinds):
        if k == "periodic":
            out.append(PERIODIC_SELF[f])
        else:
            vals = ""
            if k == "inlet":
                vals = " " + " ".join(_fmt(v) for v in values[f])
            out.append(f"-1 {ids[k]}{vals}")
    return out


def prim_to_q(prim, jac, gamma):
    """U/J from primitives, with the arithmetic of block::initialQ (src/block.cpp:554-563)."""
    rho, u, v, w, p = prim
    rhoe = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho / jac, (rho * u) / jac, (rho * v) / jac, (rho * w) / jac, rhoe / jac])


def reset_lines(text: str) -> int:
    """Cells whose energy the reference's con2prim reset: it prints one "negative pressure
    at<rank>:i,j,k" line per cell and right-hand side (src/physicsModel.cpp:324-332)."""
    return text.count("negative pressure at")


def spherical_riemann_prim(xc, yc, zc, radius=0.2, centre=(0.5, 0.5, 0.5)):
    """Spherical discontinuity: rho, p = 1, 10 inside r < radius; 0.125, 0.1 outside; u = 0."""
    dx = xc - centre[0]
    dy = yc - centre[1]
    dz = zc - centre[2]
    inside = (dx * dx + dy * dy + dz * dz) < radius * radius
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 10.0, 0.1)
    zero = np.zeros_like(rho)
    return np.stack([rho, zero, zero, zero, p])
