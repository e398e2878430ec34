"""Generate the golden fixtures in tests/golden/ by running the NUC3d reference.

    make -C oracle ref && python tests/golden/make_golden.py [--diag] [case ...]

Needs the reference binaries built under oracle/_ref (from the reference sources);
the fixtures it writes are committed so the tests never need the sources.
Each fixture <name>.npz holds one case:
  config (json)   scheme/model/physics/BC description, mesh recipe
  q0              Q = U/J at t = 0 (5, nz, ny, nx)
  rhs, dt_local   one right-hand side at q0 (EulerData3D::solve / its NS override)
  q1, qn          Q after 1 and after `nsteps` TVD-RK3 steps (block::solve)
  dt, time, res   per-step dt, accumulated time and residual (block::RES) of those nsteps
  reset_cells     con2prim energy resets over the nsteps (its printed lines)
  metrics_*       (only in the first fixture) the reference's metrics, to pin the
                  host metric computation
multi/<name>.2ranks.npz the same case run as two ranks (cases marked ranks2), and
diag/<name>.npz the postproc::solveQ diagnostics of the state after those n steps
(--diag regenerates only these; diag/tgv_ns_weno5js_lf.2ranks.npz is the same case run
as two ranks, to pin the sum over blocks).
Node coordinates use only + - * / (oracle.refrun.box_nodes), so tests rebuild the
mesh bit for bit instead of storing it.
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import refrun as R  # noqa: E402

OUT = Path(__file__).resolve().parent

TWO_PI = 2.0 * math.pi


def case_defs():
    """Small non-cubic cases covering every scheme, splitting and BC of the hot path."""
    return [
        dict(name="tgv_ns_weno5js_lf", model="NavierStokes3d", riemann="LF",
             schemes=("weno5js",) * 3, shape=(16, 12, 8), lo=(0, 0, 0), hi=(TWO_PI,) * 3,
             wavy=0.0, faces=["periodic"] * 6, init="tgv",
             params=dict(Reynolds=1600.0, Mach=0.1, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=5, metrics=True),
        dict(name="sphere_euler_weno5z_ausm_outlet", model="Euler3d", riemann="AUSM",
             schemes=("weno5z",) * 3, shape=(12, 12, 12), lo=(0, 0, 0), hi=(1, 1, 1),
             wavy=0.0, faces=["outlet"] * 6, init="sphere",
             params=dict(Reynolds=1000.0, Mach=1.0, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=5),
        dict(name="wavy_euler_weno5js_lf", model="Euler3d", riemann="LF",
             schemes=("weno5js",) * 3, shape=(16, 8, 12), lo=(0, 0, 0), hi=(2.0, 1.0, 1.5),
             wavy=0.3, faces=["periodic"] * 6, init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="bc_ns_weno7js_ausmp", model="NavierStokes3d", riemann="AUSMp",
             schemes=("weno7js",) * 3, shape=(16, 12, 12), lo=(0, 0, 0), hi=(2.0, 1.0, 1.0),
             wavy=0.2, faces=["inlet", "outlet", "wall", "symm", "periodic", "periodic"],
             init="channel",
             params=dict(Reynolds=200.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.2), nsteps=3),
        dict(name="mixed_euler_lf_outlet_symm", model="Euler3d", riemann="LF",
             schemes=("weno5js", "weno5z", "weno7js"), shape=(12, 12, 12), lo=(0, 0, 0),
             hi=(1.0, 1.0, 1.0), wavy=0.25,
             faces=["outlet", "outlet", "periodic", "periodic", "symm", "symm"], init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.8, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="ns_ausm_weno5z_wall_inlet", model="NavierStokes3d", riemann="AUSM",
             schemes=("weno5z",) * 3, shape=(12, 12, 16), lo=(0, 0, 0), hi=(1.0, 1.0, 2.0),
             wavy=0.0, faces=["periodic", "periodic", "wall", "wall", "inlet", "outlet"],
             init="channel",
             params=dict(Reynolds=300.0, Mach=0.6, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.1), nsteps=3),
        dict(name="crweno5_euler_lf_periodic", model="Euler3d", riemann="LF",
             schemes=("crweno5",) * 3, shape=(16, 12, 12), lo=(0, 0, 0), hi=(2.0, 1.0, 1.0),
             wavy=0.2, faces=["periodic"] * 6, init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="hccs_ns_ausm_bc", model="NavierStokes3d", riemann="AUSM",
             schemes=("hccs",) * 3, shape=(16, 12, 12), lo=(0, 0, 0), hi=(2.0, 1.0, 1.0),
             wavy=0.15, faces=["inlet", "outlet", "wall", "symm", "periodic", "periodic"],
             init="channel",
             params=dict(Reynolds=200.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.2), nsteps=3),
        dict(name="weno3js_euler_lf_bc", model="Euler3d", riemann="LF",
             schemes=("weno3js",) * 3, shape=(16, 12, 12), lo=(0, 0, 0), hi=(2.0, 1.0, 1.0),
             wavy=0.2, faces=["inlet", "outlet", "wall", "symm", "periodic", "periodic"],
             init="channel",
             params=dict(Reynolds=1000.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="upwind1st_euler_ausm", model="Euler3d", riemann="AUSM",
             schemes=("upwind1st",) * 3, shape=(12, 16, 12), lo=(0, 0, 0), hi=(1.0, 1.5, 1.0),
             wavy=0.15, faces=["periodic", "periodic", "outlet", "outlet", "symm", "symm"],
             init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.8, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="mixed_low_order_ausmp", model="Euler3d", riemann="AUSMp",
             schemes=("weno3js", "upwind1st", "weno5z"), shape=(16, 12, 12), lo=(0, 0, 0),
             hi=(2.0, 1.0, 1.0), wavy=0.2,
             faces=["outlet", "outlet", "periodic", "periodic", "wall", "symm"], init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.6, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="ns_cd2_weno5z_bc", model="NavierStokes3d", riemann="AUSM",
             schemes=("weno5z",) * 3, vis=("cd2",) * 3, shape=(16, 12, 12), lo=(0, 0, 0),
             hi=(2.0, 1.0, 1.0), wavy=0.2,
             faces=["inlet", "outlet", "wall", "symm", "periodic", "periodic"], init="channel",
             params=dict(Reynolds=200.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.2), nsteps=3),
        dict(name="ns_cd8_weno7js_lf", model="NavierStokes3d", riemann="LF",
             schemes=("weno7js",) * 3, vis=("cd8",) * 3, shape=(16, 16, 12), lo=(0, 0, 0),
             hi=(2.0, 1.0, 1.0), wavy=0.15,
             faces=["periodic", "periodic", "wall", "outlet", "inlet", "symm"], init="channel",
             params=dict(Reynolds=300.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.1), nsteps=3),
        dict(name="ns_mixed_vis_ausmp", model="NavierStokes3d", riemann="AUSMp",
             schemes=("weno7js", "weno5js", "hccs"), vis=("cd8", "cd2", "cd6"),
             shape=(16, 12, 16), lo=(0, 0, 0), hi=(2.0, 1.0, 1.5), wavy=0.2,
             faces=["inlet", "outlet", "periodic", "periodic", "wall", "symm"], init="channel",
             params=dict(Reynolds=250.0, Mach=0.5, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.1), nsteps=3),
        dict(name="tgv_ns_hccs77_lf", model="NavierStokes3d", riemann="LF",
             schemes=("hccs77",) * 3, shape=(16, 12, 12), lo=(0, 0, 0), hi=(TWO_PI,) * 3,
             wavy=0.0, faces=["periodic"] * 6, init="tgv",
             params=dict(Reynolds=1600.0, Mach=0.1, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
        dict(name="mixed_hccs77_euler_ausmp", model="Euler3d", riemann="AUSMp",
             schemes=("hccs77", "weno5z", "hccs77"), shape=(24, 12, 12), lo=(0, 0, 0),
             hi=(1.0, 1.0, 1.0), wavy=0.2,
             faces=["periodic", "periodic", "outlet", "symm", "periodic", "periodic"],
             init="sphere",
             params=dict(Reynolds=1000.0, Mach=1.0, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3, ranks2=True),
        # con2prim's energy reset (src/physicsModel.cpp:324-332): the blast trips it at stages
        # 1 and 2 of the first step, and cells planted with negative internal energy trip it
        # at stage 0, where the reset state is what Q_Euler keeps (src/PDEData3d.cpp:74-76)
        dict(name="sphere_reset_euler_weno5z_ausm", model="Euler3d", riemann="AUSM",
             schemes=("weno5z",) * 3, shape=(24, 24, 24), lo=(0, 0, 0), hi=(1, 1, 1),
             wavy=0.0, faces=["outlet"] * 6, init="sphere_reset",
             params=dict(Reynolds=1000.0, Mach=1.0, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3, diag=False),
        dict(name="mixed_compact_ausmp", model="Euler3d", riemann="AUSMp",
             schemes=("crweno5", "hccs", "weno5z"), shape=(12, 16, 12), lo=(0, 0, 0),
             hi=(1.0, 1.5, 1.0), wavy=0.2,
             faces=["periodic", "periodic", "outlet", "outlet", "symm", "symm"], init="smooth",
             params=dict(Reynolds=1000.0, Mach=0.8, Pt=0.72, Gamma=1.4, T_ref=110.4,
                         T_inf=288.0, T_wall=1.0), nsteps=3),
    ]


def inlet_state(p):
    g, m = p["Gamma"], p["Mach"]
    return [1.0, 0.5, 0.0, 0.0, 1.0 / (g * m * m)]


def initial_prim(kind, xc, yc, zc, p):
    g, m = p["Gamma"], p["Mach"]
    if kind == "sphere":
        return R.spherical_riemann_prim(xc, yc, zc)
    if kind == "sphere_reset":
        # the blast, plus moving cells with negative pressure (so negative internal energy)
        # on a sparse lattice outside the sphere
        prim = R.spherical_riemann_prim(xc, yc, zc)
        n = xc.shape
        k, j, i = np.meshgrid(*(np.arange(m) for m in n), indexing="ij")
        plant = ((i % 11 == 3) & (j % 13 == 5) & (k % 7 == 2))
        plant &= (xc - 0.5) ** 2 + (yc - 0.5) ** 2 + (zc - 0.5) ** 2 > 0.3 ** 2
        prim[1] = np.where(plant, 0.5, prim[1])
        prim[3] = np.where(plant, -0.25, prim[3])
        prim[4] = np.where(plant, -0.01, prim[4])
        return prim
    if kind == "smooth":
        rho = 1.0 + 0.2 * np.sin(2.0 * math.pi * xc) * np.cos(math.pi * yc)
        u = 0.3 + 0.1 * np.cos(math.pi * zc)
        v = 0.1 * np.sin(math.pi * xc)
        w = -0.05 * np.cos(2.0 * math.pi * yc)
        pr = 1.0 / (g * m * m) * (1.0 + 0.1 * np.sin(math.pi * zc))
        return np.stack([rho, u, v, w, pr])
    if kind == "channel":
        rho = 1.0 + 0.05 * np.sin(math.pi * xc) * np.sin(math.pi * yc)
        u = 0.5 * (1.0 + 0.1 * np.cos(math.pi * zc))
        v = 0.02 * np.sin(2.0 * math.pi * xc)
        w = 0.01 * np.cos(math.pi * yc)
        pr = 1.0 / (g * m * m) * (1.0 + 0.02 * np.cos(math.pi * xc))
        return np.stack([rho, u, v, w, pr])
    raise ValueError(kind)


def build_case(cd):
    nx, ny, nz = cd["shape"]
    x, y, z = R.box_nodes(nx, ny, nz, lo=cd["lo"], hi=cd["hi"], wavy=cd["wavy"])
    inlet = inlet_state(cd["params"])
    values = [inlet if f == "inlet" else None for f in cd["faces"]]
    bc = R.bc_lines(cd["faces"], values)
    case = R.Case(model=cd["model"], riemann=cd["riemann"], schemes=cd["schemes"],
                  vis=tuple(cd.get("vis", ("cd6",) * 3)),
                  params=cd["params"], nodes=[(x, y, z)], bc_topo=[bc],
                  benchmark=2 if cd["init"] == "tgv" else 0)
    return case


def generate(cd):
    case = build_case(cd)
    init = R.run(case, "init")[0]
    if cd["init"] != "tgv":
        xc, yc, zc = (init[f"xyz_center.{i}"] for i in range(3))
        prim = initial_prim(cd["init"], xc, yc, zc, cd["params"])
        q0 = R.prim_to_q(prim, init["jac"], cd["params"]["Gamma"])
        case.start_step = 1
        case.q0 = [q0]
    else:
        q0 = R.stack(init, "Q", 5)
    rhs = R.run(case, "rhs")[0]
    s1 = R.run(case, "steps", 1)[0]
    printed = []
    sn = R.run(case, "steps", cd["nsteps"], stdout=printed)[0]
    out = dict(
        config=json.dumps({k: v for k, v in cd.items()}),
        q0=q0, rhs=R.stack(rhs, "RHS", 5), dt_local=rhs["dt_local"],
        q1=R.stack(s1, "Q", 5), qn=R.stack(sn, "Q", 5), dt=sn["dt"], time=sn["time"],
        res=sn["res"],  # block::RES after each step (PDEData3d::setRES)
        # cells whose energy con2prim reset over the n steps (one printed line each)
        reset_cells=np.array([R.reset_lines(printed[0])]),
    )
    if cd.get("metrics"):
        out["metrics_jac"] = init["jac"]
        for nm in ("xi_xyz", "eta_xyz", "zeta_xyz"):
            out[f"metrics_{nm}"] = R.stack(init, nm, 3)
        out["metrics_dxyz"] = np.stack([init[f"{a}.{i}"] for a in ("dx", "dy", "dz")
                                        for i in range(3)])
    # stock glibc pow versus the correctly rounded pow of the oracle build
    libm = R.run(case, "steps", cd["nsteps"], binary="nuc3d_ref_libm_taps")[0] \
        if (R.REF_BIN_DIR / "nuc3d_ref_libm_taps").exists() else None
    if libm is not None:
        qa, qb = R.stack(libm, "Q", 5), out["qn"]
        out["libm_max_rel_diff"] = np.array([np.max(np.abs(qa - qb)) / np.max(np.abs(qb))])
    np.savez_compressed(OUT / f"{cd['name']}.npz", **out)
    return out


DIAG = OUT / "diag"
MULTI = OUT / "multi"


def generate_two_ranks(cd, q0):
    """The case as two ranks cut in half along xi (periodic xi faces), run for its n
    steps: multi/<name>.2ranks.npz holds Q of both ranks side by side.  For hccs77 this
    is not the one-rank result: each block solves its own system with explicit rows at
    the cut."""
    case = build_case(cd)
    if cd["init"] != "tgv":
        h = cd["shape"][0] // 2
        case.q0 = [q0[..., :h], q0[..., h:]]
        case.start_step = 1
    case = split_xi(case, cd)
    out = R.run(case, "steps", cd["nsteps"])
    MULTI.mkdir(exist_ok=True)
    res = dict(nsteps=np.array([cd["nsteps"]]), q0=q0,
               qn=np.concatenate([R.stack(o, "Q", 5) for o in out], axis=-1),
               dt=out[0]["dt"], time=out[0]["time"], res=out[0]["res"])
    np.savez_compressed(MULTI / f"{cd['name']}.2ranks.npz", **res)
    return res


def split_xi(case, cd):
    """The case as two ranks, the xi range cut in half (periodic xi faces only); the
    other faces keep their kind (periodic ones join the rank to itself)."""
    (x, y, z), = case.nodes
    h = cd["shape"][0] // 2
    nodes = [tuple(a[:, :, :h + 1] for a in (x, y, z)), tuple(a[:, :, h:] for a in (x, y, z))]
    topo = []
    for r in range(2):
        lines = [f"{1 - r} 1", f"{1 - r} 0"]
        lines += [f"{r} {f ^ 1}" if cd["faces"][f] == "periodic" else case.bc_topo[0][f]
                  for f in range(2, 6)]
        topo.append(lines)
    case.nodes, case.bc_topo = nodes, topo
    return case


TILESIZE = {"weno7js": 4, "hccs": 4, "hccs77": 4, "weno3js": 2, "upwind1st": 1}
VIS_REACH = {"cd2": 1, "cd6": 3, "cd8": 4}


def diag_defined(cd):
    """The difference operator's inner loop starts at the scheme's tilesize; a stencil that
    reaches further reads outside the reference's rows (src/centraldifference6th.cpp:26-43)."""
    vis = cd.get("vis", ("cd6",) * 3)
    return all(TILESIZE.get(cd["schemes"][d], 3) >= VIS_REACH[vis[d]] for d in range(3))


def generate_diag(cd, nranks=1):
    """postproc::solveQ after the case's n steps (block::Post, src/block.cpp:601-618):
    enstrophy and kinetic-energy totals, and the per-cell vorticity (3), enstrophy
    density and Q-criterion fields."""
    case = build_case(cd)
    case.post_q = True
    if cd["init"] != "tgv":
        init = R.run(case, "init")[0]
        xc, yc, zc = (init[f"xyz_center.{i}"] for i in range(3))
        case.q0 = [R.prim_to_q(initial_prim(cd["init"], xc, yc, zc, cd["params"]), init["jac"],
                               cd["params"]["Gamma"])]
        case.start_step = 1
    if nranks == 2:
        case = split_xi(case, cd)
    out = R.run(case, "post", cd["nsteps"])
    cat = lambda key: np.concatenate([d[key] for d in out], axis=-1)  # noqa: E731
    res = dict(
        nsteps=np.array([cd["nsteps"]]), nranks=np.array([nranks]),
        enstrophy=out[0]["enstrophy_glb"], kinetic=out[0]["kinetic_glb"],
        fields=np.stack([cat(f"qfield.{k}") for k in range(9, 14)]),
    )
    DIAG.mkdir(exist_ok=True)
    tag = "" if nranks == 1 else f".{nranks}ranks"
    np.savez_compressed(DIAG / f"{cd['name']}{tag}.npz", **res)
    return res


def main(names=None, diag_only=False):
    for cd in case_defs():
        if names and cd["name"] not in names:
            continue
        if not diag_only:
            o = generate(cd)
            extra = f" libm_rel_diff={o['libm_max_rel_diff'][0]:.3g}" if "libm_max_rel_diff" in o else ""
            print(f"{cd['name']}: dt_local={o['dt_local'][0]:.6g} dt={o['dt']}{extra}")
            if cd.get("ranks2"):
                t = generate_two_ranks(cd, o["q0"])
                print(f"{cd['name']} 2 ranks: dt={t['dt']}")
        if not cd.get("diag", True):
            continue
        if not diag_defined(cd):
            print(f"{cd['name']} diag: skipped (the reference's difference reads past its tile)")
            continue
        d = generate_diag(cd)
        print(f"{cd['name']} diag: enstrophy={d['enstrophy'][0]:.12g} kinetic={d['kinetic'][0]:.12g}")
        if cd["name"] == "tgv_ns_weno5js_lf":
            d = generate_diag(cd, nranks=2)
            print(f"{cd['name']} diag 2 ranks: enstrophy={d['enstrophy'][0]:.12g}")


if __name__ == "__main__":
    args = sys.argv[1:]
    main([a for a in args if a != "--diag"], diag_only="--diag" in args)
