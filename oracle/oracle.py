"""ctypes view of the C restatement (oracle/_ref/liboracle.so, built from nuc3d_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker of the GPU path; nothing in the product imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "liboracle.so"
SCHEMES = {"weno5js": 0, "weno5z": 1, "weno7js": 2, "crweno5": 3, "hccs": 4, "weno3js": 5,
           "upwind1st": 6, "hccs77": 7}
VIS = {"cd6": 0, "cd2": 1, "cd8": 2}
RIEMANN = {"LF": 0, "AUSM": 1, "AUSMp": 2}
MODELS = {"Euler3d": 0, "NavierStokes3d": 1}


class OcConfig(ctypes.Structure):
    _fields_ = [("scheme", ctypes.c_int * 3), ("riemann", ctypes.c_int), ("model", ctypes.c_int),
                ("compat", ctypes.c_int), ("vis", ctypes.c_int * 3)] + [
        (k, ctypes.c_double) for k in ("gamma", "mach", "reynolds", "prandtl", "t_ref", "t_inf",
                                       "t_wall", "cfl")]


class OcBlock(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("bc_type", ctypes.c_int * 6), ("bc_id", ctypes.c_int * 6),
                ("bcv", ctypes.c_double * 30)] + [
        (k, ctypes.c_void_p) for k in ("jac", "xi", "eta", "zeta", "dxyz", "q", "rhs")]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            subprocess.run(["make", "-C", str(HERE), "oracle"], check=True, capture_output=True)
        _lib = ctypes.CDLL(str(LIB))
        _lib.oc_rhs.argtypes = [ctypes.POINTER(OcConfig), ctypes.c_int, ctypes.POINTER(OcBlock),
                                ctypes.POINTER(ctypes.c_double)]
        _lib.oc_step.argtypes = [ctypes.POINTER(OcConfig), ctypes.c_int, ctypes.POINTER(OcBlock),
                                 ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        _lib.oc_metrics.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 8
        _lib.oc_diag.argtypes = [ctypes.POINTER(OcConfig), ctypes.c_int, ctypes.POINTER(OcBlock),
                                 ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_void_p)]
        _lib.oc_cr_pow.restype = ctypes.c_double
        _lib.oc_cr_pow.argtypes = [ctypes.c_double, ctypes.c_double]
    return _lib


def cr_pow(x: float, y: float) -> float:
    """The oracle's pow for the energy reset (oracle/cr_pow.h)."""
    return lib().oc_cr_pow(x, y)


def _ptr(a):
    return a.ctypes.data if a is not None else None


def metrics(x, y, z) -> dict:
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    nz, ny, nx = (s - 1 for s in x.shape)
    sh = (nz, ny, nx)
    out = {"jac": np.empty(sh), "xi_xyz": np.empty((3,) + sh), "eta_xyz": np.empty((3,) + sh),
           "zeta_xyz": np.empty((3,) + sh), "dxyz": np.empty((9,) + sh)}
    rc = lib().oc_metrics(nx, ny, nz, _ptr(x), _ptr(y), _ptr(z), _ptr(out["jac"]),
                          _ptr(out["xi_xyz"]), _ptr(out["eta_xyz"]), _ptr(out["zeta_xyz"]),
                          _ptr(out["dxyz"]))
    if rc:
        raise ValueError("cells per axis must be multiples of 4")
    return out


class Run:
    """A set of blocks (metrics, BCs, state) advanced by the restatement."""

    def __init__(self, scheme, riemann, model, params, cfl=0.5, compat=True, vis=("cd6",) * 3):
        c = OcConfig()
        for d in range(3):
            c.scheme[d] = SCHEMES[scheme[d]]
            c.vis[d] = VIS[vis[d]]
        c.riemann, c.model, c.compat = RIEMANN[riemann], MODELS[model], int(compat)
        c.gamma, c.mach, c.reynolds = params["Gamma"], params["Mach"], params["Reynolds"]
        c.prandtl, c.t_ref, c.t_inf = params["Pt"], params["T_ref"], params["T_inf"]
        c.t_wall, c.cfl = params["T_wall"], cfl
        self.cfg = c
        self.blocks = []
        self._keep = []

    def add_block(self, m: dict, bc_type, bc_id, bc_values, q):
        b = OcBlock()
        sh = m["jac"].shape
        b.n[0], b.n[1], b.n[2] = sh[2], sh[1], sh[0]
        for f in range(6):
            b.bc_type[f], b.bc_id[f] = int(bc_type[f]), int(bc_id[f])
            if self.cfg.scheme[f // 2] == SCHEMES["hccs77"] and int(bc_type[f]) == -1:
                raise ValueError("hccs77 is defined for neighbour faces only "
                                 "(src/fieldOperator.cpp:400-412, src/hccs77.cpp:570-590)")
        vals = np.zeros(30) if bc_values is None else np.asarray(bc_values, dtype=np.float64).ravel()
        for i in range(30):
            b.bcv[i] = vals[i]
        arrs = {k: np.ascontiguousarray(m[k], dtype=np.float64)
                for k in ("jac", "xi_xyz", "eta_xyz", "zeta_xyz", "dxyz")}
        qq = np.array(q, dtype=np.float64, copy=True)
        rhs = np.zeros_like(qq)
        b.jac, b.xi, b.eta = _ptr(arrs["jac"]), _ptr(arrs["xi_xyz"]), _ptr(arrs["eta_xyz"])
        b.zeta, b.dxyz, b.q, b.rhs = _ptr(arrs["zeta_xyz"]), _ptr(arrs["dxyz"]), _ptr(qq), _ptr(rhs)
        self._keep.append((arrs, qq, rhs))
        self.blocks.append(b)
        return len(self.blocks) - 1

    def _arr(self):
        return (OcBlock * len(self.blocks))(*self.blocks)

    def rhs(self):
        arr = self._arr()
        dt = ctypes.c_double()
        lib().oc_rhs(ctypes.byref(self.cfg), len(self.blocks), arr, ctypes.byref(dt))
        return dt.value, [k[2].copy() for k in self._keep]

    def step(self, n):
        """n steps: (dt per step, time); self.res gets the residual of each step."""
        arr = self._arr()
        dts = (ctypes.c_double * n)()
        res = (ctypes.c_double * n)()
        t = ctypes.c_double(0.0)
        lib().oc_step(ctypes.byref(self.cfg), len(self.blocks), arr, n, dts, ctypes.byref(t), res)
        self.res = np.array(res[:])
        return np.array(dts[:]), t.value

    def q(self, b):
        return self._keep[b][1]

    def diag(self):
        """postproc::solveQ of the current state: (enstrophy, kinetic, per-block fields of
        shape (5, nz, ny, nx): vorticity x, y, z, enstrophy density, Q)."""
        arr = self._arr()
        fields = [np.empty((5,) + k[0]["jac"].shape) for k in self._keep]
        ptrs = (ctypes.c_void_p * len(fields))(*[f.ctypes.data for f in fields])
        ens, kin = ctypes.c_double(), ctypes.c_double()
        lib().oc_diag(ctypes.byref(self.cfg), len(self.blocks), arr, ctypes.byref(ens),
                      ctypes.byref(kin), ptrs)
        return ens.value, kin.value, fields
