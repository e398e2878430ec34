"""nuc3d_b200 -- NUC3d's per-block right-hand side and TVD-RK3 update on one B200.

Python view of the C ABI in include/nuc3d_gpu.h (libnuc3d_b200.so, built in-tree
by ``python -m nuc3d_b200.build``).  The configuration mirrors the reference's
input files: ``Config.scheme_ivs``/``scheme_vis`` are Method.in's
scheme_{x,y,z}_ivs/_vis (src/fieldOperator.cpp:20-33), ``riemann``/``model`` and
the physical constants are PhysModel.in (src/physicsModel.cpp:41-69), ``cfl`` is
IOController.in's (src/IOcontroller.cpp:22-29).  A block is described the way
BC_Topo_<rank>.in does it (src/boundaryConditions.cpp:69-93).

There is no CPU path: importing this package without the built library raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .metrics import metrics_from_nodes  # noqa: F401  (host-side block::getJacobians)

import os

# NUC3D_LIB selects another build of the library (e.g. a variant compiled with
# different tile options); by default the in-tree build is used.
_LIB_PATH = Path(os.environ.get("NUC3D_LIB") or Path(__file__).resolve().parent / "libnuc3d_b200.so")

NUC3D_OK, NUC3D_EINVAL, NUC3D_ECUDA, NUC3D_ESTATE, NUC3D_ENUMERIC, NUC3D_ENOTSUP = range(6)
ST_NEG_PRESSURE, ST_ENERGY_RESET, ST_NONFINITE = 1, 2, 4
BC_INLET, BC_OUTLET, BC_WALL, BC_SYMM = 0, 1, 2, 3

EXPORTED = (
    "nuc3d_last_error", "nuc3d_create", "nuc3d_destroy", "nuc3d_block_add",
    "nuc3d_block_set_metrics", "nuc3d_finalize", "nuc3d_block_set_q", "nuc3d_block_get_q",
    "nuc3d_block_q_device", "nuc3d_rhs", "nuc3d_block_get_rhs", "nuc3d_step", "nuc3d_solve_host",
    "nuc3d_sync",
    "nuc3d_get_time", "nuc3d_set_time", "nuc3d_get_status", "nuc3d_set_stream",
    "nuc3d_use_graph", "nuc3d_block_get_prim", "nuc3d_block_get_vis", "nuc3d_profile_sweep",
    "nuc3d_rhs_noalloc", "nuc3d_kernels_per_step", "nuc3d_diagnostics", "nuc3d_block_get_diag",
    "nuc3d_block_set_nodes", "nuc3d_block_get_metrics", "nuc3d_sensor_record",
    "nuc3d_sensor_loss_grad", "nuc3d_sensor_adam", "nuc3d_set_sensor", "nuc3d_set_tiles",
    "nuc3d_get_tiles", "nuc3d_autotune", "nuc3d_get_energy_resets", "nuc3d_set_pipeline",
    "nuc3d_get_pipeline", "nuc3d_rhs_stage", "nuc3d_rk_stage", "nuc3d_get_residual",
    "nuc3d_set_compact_solver", "nuc3d_get_compact_solver", "nuc3d_set_sensor_theta",
    "nuc3d_debug_get", "nuc3d_set_host_pipeline", "nuc3d_get_host_pipeline",
)


def fp64_peak_tflops(device: int = 0, reps: int = 20) -> float:
    """Measured FP64 FMA throughput of the device (libnuc3d_probe.so microbenchmark)."""
    p = _LIB_PATH.with_name("libnuc3d_probe.so")
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m nuc3d_b200.build`")
    lib = ctypes.CDLL(str(p))
    lib.nuc3d_probe_fp64_tflops.restype = ctypes.c_double
    lib.nuc3d_probe_fp64_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    v = lib.nuc3d_probe_fp64_tflops(device, reps)
    if v < 0:
        raise RuntimeError(f"fp64 probe failed ({v})")
    return v


class Nuc3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nuc3d error {code}: {msg}")
        self.code = code


class _Cfg(ctypes.Structure):
    _fields_ = [
        ("scheme_ivs", ctypes.c_char_p * 3),
        ("scheme_vis", ctypes.c_char_p * 3),
        ("riemann", ctypes.c_char_p),
        ("model", ctypes.c_char_p),
        ("reynolds", ctypes.c_double), ("mach", ctypes.c_double), ("prandtl", ctypes.c_double),
        ("gamma", ctypes.c_double), ("t_ref", ctypes.c_double), ("t_inf", ctypes.c_double),
        ("t_wall", ctypes.c_double), ("cfl", ctypes.c_double),
        ("exact", ctypes.c_int), ("weno5z_compat", ctypes.c_int),
    ]


_lib = None


def load_library() -> ctypes.CDLL:
    """The CUDA library; raises if it was not built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m nuc3d_b200.build`")
    lib = ctypes.CDLL(str(_LIB_PATH))
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    PD = ctypes.POINTER(ctypes.c_double)
    lib.nuc3d_last_error.restype = ctypes.c_char_p
    lib.nuc3d_create.argtypes = [ctypes.POINTER(_Cfg), I, ctypes.POINTER(P)]
    lib.nuc3d_destroy.argtypes = [P]
    lib.nuc3d_block_add.argtypes = [P, I, I, I, ctypes.POINTER(I), ctypes.POINTER(I), PD,
                                    ctypes.POINTER(I)]
    lib.nuc3d_block_set_metrics.argtypes = [P, I, PD, PD, PD, PD, PD]
    lib.nuc3d_finalize.argtypes = [P]
    lib.nuc3d_block_set_q.argtypes = [P, I, P]
    lib.nuc3d_block_get_q.argtypes = [P, I, P]
    lib.nuc3d_block_q_device.argtypes = [P, I, ctypes.POINTER(P)]
    lib.nuc3d_rhs.argtypes = [P, PD]
    lib.nuc3d_block_get_rhs.argtypes = [P, I, PD]
    lib.nuc3d_step.argtypes = [P, I]
    lib.nuc3d_solve_host.argtypes = [P, ctypes.POINTER(P), I]
    lib.nuc3d_set_tiles.argtypes = [P, ctypes.POINTER(I)]
    lib.nuc3d_get_tiles.argtypes = [P, ctypes.POINTER(I)]
    lib.nuc3d_autotune.argtypes = [P, I, ctypes.POINTER(I), PD]
    lib.nuc3d_sync.argtypes = [P]
    lib.nuc3d_get_time.argtypes = [P, PD, PD]
    lib.nuc3d_set_time.argtypes = [P, D]
    lib.nuc3d_get_status.argtypes = [P, ctypes.POINTER(ctypes.c_uint)]
    lib.nuc3d_get_energy_resets.argtypes = [P, ctypes.POINTER(ctypes.c_ulonglong)]
    lib.nuc3d_set_pipeline.argtypes = [P, I]
    lib.nuc3d_get_pipeline.argtypes = [P, ctypes.POINTER(I)]
    lib.nuc3d_set_compact_solver.argtypes = [P, I]
    lib.nuc3d_set_sensor_theta.argtypes = [P, ctypes.c_float]
    lib.nuc3d_debug_get.argtypes = [P, I, I, PD]
    lib.nuc3d_set_host_pipeline.argtypes = [P, I]
    lib.nuc3d_get_host_pipeline.argtypes = [P, ctypes.POINTER(I)]
    lib.nuc3d_get_compact_solver.argtypes = [P, ctypes.POINTER(I)]
    lib.nuc3d_rhs_stage.argtypes = [P, I, PD]
    lib.nuc3d_rk_stage.argtypes = [P, I, D]
    lib.nuc3d_get_residual.argtypes = [P, PD]
    lib.nuc3d_set_stream.argtypes = [P, P]
    lib.nuc3d_use_graph.argtypes = [P, I]
    lib.nuc3d_block_get_prim.argtypes = [P, I, PD]
    lib.nuc3d_block_get_vis.argtypes = [P, I, PD]
    lib.nuc3d_profile_sweep.argtypes = [P, I, I, PD]
    PI = ctypes.POINTER(I)
    lib.nuc3d_kernels_per_step.argtypes = [P, PI]
    lib.nuc3d_diagnostics.argtypes = [P, PD, PD]
    lib.nuc3d_block_set_nodes.argtypes = [P, I, PD, PD, PD]
    ULL = ctypes.c_ulonglong
    lib.nuc3d_sensor_record.argtypes = [P, I, P, P, P, ULL, ctypes.POINTER(ULL)]
    F = ctypes.c_float
    lib.nuc3d_sensor_loss_grad.argtypes = [P, P, P, ctypes.c_longlong, F, P, P, P, P]
    lib.nuc3d_sensor_adam.argtypes = [P, P, P, P, F, F, F, F, I, P]
    lib.nuc3d_set_sensor.argtypes = [P, ctypes.POINTER(F), F]
    lib.nuc3d_block_get_metrics.argtypes = [P, I, PD, PD, PD, PD, PD]
    lib.nuc3d_block_get_diag.argtypes = [P, I, PD]
    lib.nuc3d_rhs_noalloc.argtypes = [ctypes.POINTER(_Cfg), I, I, I, I, PI, PI, PD, P, P, P, P,
                                      P, P, P, PD, P]
    for name in EXPORTED:
        if name != "nuc3d_last_error":
            getattr(lib, name).restype = ctypes.c_int
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != NUC3D_OK:
        raise Nuc3dError(rc, load_library().nuc3d_last_error().decode())


def _pd(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Config:
    """Method.in + PhysModel.in + cfl of the reference."""

    scheme_ivs: tuple = ("weno5js", "weno5js", "weno5js")
    scheme_vis: tuple = ("cd6", "cd6", "cd6")
    riemann: str = "LF"
    model: str = "Euler3d"
    reynolds: float = 1000.0
    mach: float = 0.5
    prandtl: float = 0.72
    gamma: float = 1.4
    t_ref: float = 110.4
    t_inf: float = 288.0
    t_wall: float = 1.0
    cfl: float = 0.5
    exact: bool = True
    weno5z_compat: bool = True

    def _c(self) -> _Cfg:
        c = _Cfg()
        for d in range(3):
            c.scheme_ivs[d] = self.scheme_ivs[d].encode()
            c.scheme_vis[d] = self.scheme_vis[d].encode()
        c.riemann = self.riemann.encode()
        c.model = self.model.encode()
        for k in ("reynolds", "mach", "prandtl", "gamma", "t_ref", "t_inf", "t_wall", "cfl"):
            setattr(c, k, float(getattr(self, k)))
        c.exact = int(bool(self.exact))
        c.weno5z_compat = int(bool(self.weno5z_compat))
        return c


@dataclass
class BlockSpec:
    shape: tuple                      # (nx, ny, nz) cells
    bc_type: tuple                    # 6 faces: -1 physical, else neighbour block index
    bc_id: tuple                      # physical BC id or neighbour face
    bc_values: np.ndarray | None = None  # (6, 5) inlet primitive states
    dims: tuple = field(init=False)

    def __post_init__(self):
        self.dims = tuple(int(x) for x in self.shape)


class Solver:
    """One context: a set of blocks advanced together on one GPU."""

    def __init__(self, cfg: Config, device: int = 0):
        self.lib = load_library()
        self.cfg = cfg
        self._ctx = ctypes.c_void_p()
        self._cfg_c = cfg._c()
        _check(self.lib.nuc3d_create(ctypes.byref(self._cfg_c), device, ctypes.byref(self._ctx)))
        self.blocks: list[tuple] = []

    # -- set-up ---------------------------------------------------------------
    def add_block(self, nx, ny, nz, bc_type, bc_id, bc_values=None) -> int:
        t = (ctypes.c_int * 6)(*[int(x) for x in bc_type])
        i = (ctypes.c_int * 6)(*[int(x) for x in bc_id])
        vals = None
        if bc_values is not None:
            vals = _f64(bc_values).reshape(30)
            self._keep = vals
        out = ctypes.c_int()
        _check(self.lib.nuc3d_block_add(self._ctx, nx, ny, nz, t, i,
                                        _pd(vals) if vals is not None else None,
                                        ctypes.byref(out)))
        self.blocks.append((nx, ny, nz))
        return out.value

    def set_metrics(self, b, jac, xi_xyz, eta_xyz, zeta_xyz, dxyz=None) -> None:
        arrs = [_f64(a) for a in (jac, xi_xyz, eta_xyz, zeta_xyz)]
        dx = _f64(dxyz) if dxyz is not None else None
        _check(self.lib.nuc3d_block_set_metrics(self._ctx, b, *[_pd(a) for a in arrs],
                                                _pd(dx) if dx is not None else None))

    def set_mesh(self, b, x, y, z) -> dict:
        """Metrics of block b from its node coordinates (block::getJacobians)."""
        m = metrics_from_nodes(x, y, z)
        self.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
        return m

    def set_nodes(self, b, x, y, z) -> None:
        """Metrics of block b computed on the GPU from its node coordinates
        (block::getJacobians; bitwise the host set_mesh)."""
        arrs = [_f64(a) for a in (x, y, z)]
        _check(self.lib.nuc3d_block_set_nodes(self._ctx, b, *[_pd(a) for a in arrs]))

    def get_metrics(self, b) -> dict:
        nx, ny, nz = self.blocks[b]
        sh = (nz, ny, nx)
        out = {"jac": np.empty(sh), "xi_xyz": np.empty((3,) + sh), "eta_xyz": np.empty((3,) + sh),
               "zeta_xyz": np.empty((3,) + sh)}
        _check(self.lib.nuc3d_block_get_metrics(self._ctx, b, *[_pd(out[k]) for k in
                                                ("jac", "xi_xyz", "eta_xyz", "zeta_xyz")], None))
        return out

    def finalize(self) -> None:
        _check(self.lib.nuc3d_finalize(self._ctx))

    # -- state ----------------------------------------------------------------
    def _shape5(self, b):
        nx, ny, nz = self.blocks[b]
        return (5, nz, ny, nx)

    def set_q(self, b, q) -> None:
        q = _f64(q)
        if q.shape != self._shape5(b):
            q = q.reshape(self._shape5(b))
        _check(self.lib.nuc3d_block_set_q(self._ctx, b, q.ctypes.data))
        _check(self.lib.nuc3d_sync(self._ctx))

    def set_q_ptr(self, b, host_ptr: int) -> None:
        """Asynchronous upload from a host pointer (e.g. pinned memory)."""
        _check(self.lib.nuc3d_block_set_q(self._ctx, b, ctypes.c_void_p(host_ptr)))

    def get_q(self, b) -> np.ndarray:
        out = np.empty(self._shape5(b), dtype=np.float64)
        _check(self.lib.nuc3d_block_get_q(self._ctx, b, out.ctypes.data))
        return out

    def get_q_ptr(self, b, host_ptr: int) -> None:
        _check(self.lib.nuc3d_block_get_q(self._ctx, b, ctypes.c_void_p(host_ptr)))

    def q_device_ptr(self, b) -> int:
        p = ctypes.c_void_p()
        _check(self.lib.nuc3d_block_q_device(self._ctx, b, ctypes.byref(p)))
        return p.value

    # -- evaluation -----------------------------------------------------------
    def rhs(self) -> float:
        dt = ctypes.c_double()
        _check(self.lib.nuc3d_rhs(self._ctx, ctypes.byref(dt)))
        return dt.value

    def get_rhs(self, b) -> np.ndarray:
        out = np.empty(self._shape5(b), dtype=np.float64)
        _check(self.lib.nuc3d_block_get_rhs(self._ctx, b, _pd(out)))
        return out

    def get_prim(self, b) -> np.ndarray:
        nx, ny, nz = self.blocks[b]
        out = np.empty((4, nz, ny, nx), dtype=np.float64)
        _check(self.lib.nuc3d_block_get_prim(self._ctx, b, _pd(out)))
        return out

    def get_vis(self, b) -> np.ndarray:
        nx, ny, nz = self.blocks[b]
        out = np.empty((3, 4, nz, ny, nx), dtype=np.float64)
        _check(self.lib.nuc3d_block_get_vis(self._ctx, b, _pd(out)))
        return out

    def step(self, n: int = 1, sync: bool = True) -> None:
        _check(self.lib.nuc3d_step(self._ctx, int(n)))
        if sync:
            self.sync()

    def set_host_pipeline(self, on: bool) -> None:
        """solve_host as a copy/compute pipeline over z-slabs where it applies (default)."""
        _check(self.lib.nuc3d_set_host_pipeline(self._ctx, 1 if on else 0))

    def host_pipeline(self) -> int:
        """z-slabs solve_host pipelines over (0: whole-state chunked copies)."""
        v = ctypes.c_int()
        _check(self.lib.nuc3d_get_host_pipeline(self._ctx, ctypes.byref(v)))
        return v.value

    def solve_host(self, host_ptrs, n: int = 1) -> None:
        """n steps on host arrays, in place: every step reads each block's Q from its host
        pointer (pinned memory for full speed) and writes the new Q back there."""
        if len(host_ptrs) != len(self.blocks):
            raise ValueError("one host pointer per block")
        arr = (ctypes.c_void_p * len(host_ptrs))(*[int(p) for p in host_ptrs])
        _check(self.lib.nuc3d_solve_host(self._ctx, arr, int(n)))

    def sync(self) -> None:
        _check(self.lib.nuc3d_sync(self._ctx))

    def time_dt(self) -> tuple:
        t, dt = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.nuc3d_get_time(self._ctx, ctypes.byref(t), ctypes.byref(dt)))
        return t.value, dt.value

    def set_time(self, t: float) -> None:
        _check(self.lib.nuc3d_set_time(self._ctx, float(t)))

    def status(self) -> int:
        s = ctypes.c_uint()
        _check(self.lib.nuc3d_get_status(self._ctx, ctypes.byref(s)))
        return s.value

    def rhs_stage(self, stage: int) -> float:
        """RHS of every block at the state of RK stage `stage`; returns dt_local."""
        dt = ctypes.c_double()
        _check(self.lib.nuc3d_rhs_stage(self._ctx, int(stage), ctypes.byref(dt)))
        return dt.value

    def rk_stage(self, stage: int, dt: float) -> None:
        """TVD-RK3 stage `stage` from the last rhs_stage(stage), step size dt."""
        _check(self.lib.nuc3d_rk_stage(self._ctx, int(stage), float(dt)))

    def residual(self) -> float:
        """The residual of the last step (PDEData3d::setRES), max over blocks."""
        r = ctypes.c_double()
        _check(self.lib.nuc3d_get_residual(self._ctx, ctypes.byref(r)))
        return r.value

    def set_pipeline(self, on) -> None:
        """Persistent TMA-fed sweeps on (default) or off, or an int bitmask of directions
        (bit d: direction d; values above 1); results are identical."""
        v = int(on) if not isinstance(on, bool) else (1 if on else 0)
        _check(self.lib.nuc3d_set_pipeline(self._ctx, v))

    def pipeline(self) -> int:
        """Directions (bit d) whose sweeps run pipelined (even nx, explicit schemes, switched on);
        0 for none."""
        v = ctypes.c_int()
        _check(self.lib.nuc3d_get_pipeline(self._ctx, ctypes.byref(v)))
        return v.value

    def set_compact_solver(self, fused: bool) -> None:
        """Compact-scheme line solves fused into one kernel per direction (throughput build,
        lines of at most 256 cells; the default) or rows, Thomas and faces in three."""
        _check(self.lib.nuc3d_set_compact_solver(self._ctx, 1 if fused else 0))

    def compact_solver(self) -> int:
        """Directions (bit d) whose compact scheme runs the fused line kernel."""
        v = ctypes.c_int()
        _check(self.lib.nuc3d_get_compact_solver(self._ctx, ctypes.byref(v)))
        return v.value

    def energy_resets(self) -> int:
        """Cells whose energy con2prim reset, once per cell and right-hand side, since the
        context was created (the reference prints one "negative pressure at" line each)."""
        n = ctypes.c_ulonglong()
        _check(self.lib.nuc3d_get_energy_resets(self._ctx, ctypes.byref(n)))
        return n.value

    def profile_sweep(self, direction: int, reps: int = 10) -> float:
        """Mean device milliseconds of one launch of the direction sweep kernel."""
        ms = ctypes.c_double()
        _check(self.lib.nuc3d_profile_sweep(self._ctx, direction, reps, ctypes.byref(ms)))
        return ms.value

    def diagnostics(self) -> tuple[float, float]:
        """(enstrophy, kinetic energy) totals of the current state (postproc::solveQ)."""
        e, k = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.nuc3d_diagnostics(self._ctx, ctypes.byref(e), ctypes.byref(k)))
        return e.value, k.value

    def get_diag(self, block: int):
        """Fields of the last diagnostics call, shape (5, nz, ny, nx): vorticity x, y, z,
        enstrophy density 0.5|w|^2, Q criterion."""
        out = np.empty(self._shape5(block), dtype=np.float64)
        _check(self.lib.nuc3d_block_get_diag(self._ctx, block, _pd(out)))
        return out

    def sensor_record(self, direction: int, feat_ptr: int, label_ptr: int, where_ptr: int,
                      cap: int) -> int:
        """Record face features/labels of one direction into device buffers (pointers);
        returns the number written."""
        n = ctypes.c_ulonglong()
        _check(self.lib.nuc3d_sensor_record(self._ctx, direction, ctypes.c_void_p(feat_ptr),
                                            ctypes.c_void_p(label_ptr),
                                            ctypes.c_void_p(where_ptr) if where_ptr else None,
                                            cap, ctypes.byref(n)))
        return n.value

    def set_sensor(self, params=None, logit_threshold: float = -4.0) -> None:
        """Hybrid WENO-Z with the learned face sensor (params: 1729 floats; None: plain)."""
        if params is None:
            _check(self.lib.nuc3d_set_sensor(self._ctx, None, 0.0))
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != 1729:
            raise ValueError("the sensor has 1729 parameters")
        self._sensor_keep = p
        _check(self.lib.nuc3d_set_sensor(self._ctx, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                         float(logit_threshold)))

    TAP_KINDS = ("FluxL", "FluxR", "rFluxL", "rFluxR", "df")

    def debug_get(self, block: int, kind: str, direction: int) -> np.ndarray:
        """One debug tap (nuc3d_debug_get): kind in TAP_KINDS, shaped as the reference's
        Field for that direction, (5, n_c, n_b, n_a) with n_a the line axis (+1 for the
        face values): xi (nz, ny, nx), eta (nx, nz, ny), zeta (ny, nx, nz)."""
        k = self.TAP_KINDS.index(kind)
        nx, ny, nz = self.blocks[block]
        dims = [(nz, ny, nx), (nx, nz, ny), (ny, nx, nz)][direction]
        if k in (2, 3):
            dims = dims[:2] + (dims[2] + 1,)
        out = np.empty((5,) + dims, dtype=np.float64)
        _check(self.lib.nuc3d_debug_get(self._ctx, block, 3 * k + direction, _pd(out)))
        return out

    def set_sensor_theta(self, theta_min: float) -> None:
        """Hybrid WENO-Z deciding by hccs's theta switch: linear weights where the face's
        smallest density/pressure theta is at least theta_min (set_sensor(None): plain)."""
        _check(self.lib.nuc3d_set_sensor_theta(self._ctx, float(theta_min)))

    def set_tiles(self, shape) -> None:
        """Sweep tile shape per direction: 0 = 4 x 64, 1 = 8 x 32, 2 = 2 x 128."""
        arr = (ctypes.c_int * 3)(*[int(x) for x in shape])
        _check(self.lib.nuc3d_set_tiles(self._ctx, arr))

    def get_tiles(self) -> tuple:
        arr = (ctypes.c_int * 3)()
        _check(self.lib.nuc3d_get_tiles(self._ctx, arr))
        return tuple(arr)

    def autotune(self, reps: int = 3) -> dict:
        """Time every tile shape of each direction's sweep on the current state and keep the
        fastest (cached per grid in this process).  Returns {"shape": (s0, s1, s2),
        "ms": [[ms of shape 0, 1, 2] per direction] (None where not timed)}."""
        shp = (ctypes.c_int * 3)()
        ms = (ctypes.c_double * 9)()
        _check(self.lib.nuc3d_autotune(self._ctx, int(reps), shp, ms))
        t = [[(ms[3 * d + k] if ms[3 * d + k] >= 0 else None) for k in range(3)] for d in range(3)]
        return {"shape": tuple(shp), "ms": t}

    def kernels_per_step(self) -> int:
        """Kernels one step launches (the library's own count of its launches)."""
        n = ctypes.c_int()
        _check(self.lib.nuc3d_kernels_per_step(self._ctx, ctypes.byref(n)))
        return n.value

    def use_graph(self, on: bool) -> None:
        _check(self.lib.nuc3d_use_graph(self._ctx, int(bool(on))))

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(self.lib.nuc3d_set_stream(self._ctx, ctypes.c_void_p(stream_ptr or 0)))

    def close(self) -> None:
        if self._ctx:
            self.lib.nuc3d_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
