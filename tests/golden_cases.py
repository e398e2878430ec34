"""Load the committed golden fixtures and set up the GPU solver for them."""
from __future__ import annotations

import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from oracle import refrun as R

GOLDEN = Path(__file__).resolve().parent / "golden"
FACE_IDS = {"inlet": 0, "outlet": 1, "wall": 2, "symm": 3}
PERIODIC_NEIGHBOUR_FACE = [1, 0, 3, 2, 5, 4]


@dataclass
class Golden:
    name: str
    cfg: dict
    data: dict

    def __getattr__(self, k):
        try:
            return self.data[k]
        except KeyError as e:
            raise AttributeError(k) from e


def names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def diag_names():
    """Cases with a diagnostics fixture (not the ones whose reference diagnostics read
    outside the field: low-order schemes with cd6)."""
    return sorted(p.name[:-4] for p in (GOLDEN / "diag").glob("*.npz") if p.name.count(".") == 1)


def load_diag(name: str) -> dict:
    """postproc::solveQ of the case's state after its n steps (golden/diag/<name>.npz)."""
    z = np.load(GOLDEN / "diag" / f"{name}.npz")
    return {k: z[k] for k in z.files}


def split_xi(arrays, h):
    """Cut cell arrays (..., nz, ny, nx) at i = h into two blocks."""
    return [a[..., :h] for a in arrays], [a[..., h:] for a in arrays]


# two blocks cut along xi from one periodic block: block indices and neighbour faces
TWO_BLOCK_TYPES = [[1, 1, 0, 0, 0, 0], [0, 0, 1, 1, 1, 1]]
TWO_BLOCK_IDS = [[1, 0, 3, 2, 5, 4], [1, 0, 3, 2, 5, 4]]


def two_block_bc(g: Golden, b: int):
    """BC arrays of block b (0 left, 1 right) of the case cut in half along xi: the xi
    faces join the two blocks, the other faces keep the case's (periodic ones point at
    the block itself)."""
    t, i, v = bc_arrays(g, b)
    t[0], i[0], t[1], i[1] = 1 - b, 1, 1 - b, 0
    return t, i, v


def multi_names():
    """Cases with a two-rank fixture (golden/multi/<name>.2ranks.npz)."""
    return sorted(p.name[:-len(".2ranks.npz")] for p in (GOLDEN / "multi").glob("*.2ranks.npz"))


def load_multi(name: str) -> dict:
    z = np.load(GOLDEN / "multi" / f"{name}.2ranks.npz")
    return {k: z[k] for k in z.files}


def load(name: str) -> Golden:
    z = np.load(GOLDEN / f"{name}.npz")
    data = {k: z[k] for k in z.files}
    cfg = json.loads(str(data.pop("config")))
    return Golden(name, cfg, data)


def nodes(g: Golden):
    nx, ny, nz = g.cfg["shape"]
    return R.box_nodes(nx, ny, nz, lo=g.cfg["lo"], hi=g.cfg["hi"], wavy=g.cfg["wavy"])


def inlet_state(p):
    return [1.0, 0.5, 0.0, 0.0, 1.0 / (p["Gamma"] * p["Mach"] * p["Mach"])]


def bc_arrays(g: Golden, self_index: int = 0):
    types, ids, vals = [], [], np.zeros((6, 5))
    for f, k in enumerate(g.cfg["faces"]):
        if k == "periodic":
            types.append(self_index)
            ids.append(PERIODIC_NEIGHBOUR_FACE[f])
        else:
            types.append(-1)
            ids.append(FACE_IDS[k])
            if k == "inlet":
                vals[f] = inlet_state(g.cfg["params"])
    return types, ids, vals


def vis(g: Golden) -> tuple:
    """scheme_x/y/z_vis of the case (cd6 unless the case names others)."""
    return tuple(g.cfg.get("vis", ("cd6",) * 3))


def nuc3d_config(g: Golden, exact: bool = True):
    import nuc3d_b200 as nb
    p = g.cfg["params"]
    return nb.Config(scheme_ivs=tuple(g.cfg["schemes"]), scheme_vis=vis(g), riemann=g.cfg["riemann"],
                     model=g.cfg["model"], reynolds=p["Reynolds"], mach=p["Mach"],
                     prandtl=p["Pt"], gamma=p["Gamma"], t_ref=p["T_ref"], t_inf=p["T_inf"],
                     t_wall=p["T_wall"], cfl=0.5, exact=exact, weno5z_compat=True)


def solver(g: Golden, exact: bool = True):
    import nuc3d_b200 as nb
    s = nb.Solver(nuc3d_config(g, exact))
    nx, ny, nz = g.cfg["shape"]
    t, i, v = bc_arrays(g)
    b = s.add_block(nx, ny, nz, t, i, v)
    s.set_mesh(b, *nodes(g))
    s.finalize()
    s.set_q(b, g.q0)
    return s
