#!/usr/bin/env python
"""Throughput of NUC3d's per-block RHS + TVD-RK3 update on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload turbulence24      (the 24-block Navier-Stokes grid)
    python bench.py --workload shock_turbulence|boundary_layer   (plain against hybrid)
    python bench.py --workload compact           (crweno5 / hccs: fused against three kernels)
    python bench.py --profile-case --shape 192 --sweeps 2 [--steps N] [--ns] [--hybrid]
                                                 (untimed: the command ncu captures)

Workload (one per GPU): the shock-dominated FP64 Euler case -- a 256^3 block on
[0,1]^3 with extrapolation (outlet) faces, spherical discontinuity rho,p = 1,10
inside r < 0.2 and 0.125,0.1 outside, WENO5-Z + AUSM splitting, TVD-RK3 at CFL
0.5.  The reference has no characteristic projection; splitting is component-wise
as in src/euler3d.cpp:318-330.  A step = one TVD-RK3 step (3 stages) of the block.

Metric: Mcell-RK3-steps/s = cells x steps / device seconds, summed over GPUs
(weak scaling: every GPU advances its own block; no data-path collective).
The timed state (5 x 256^3 doubles = 671 MB per buffer, 4 GB per block) is far
larger than the 126 MB L2.

--impl reference times the reference's own CPU code (oracle/_ref/nuc3d_ref_taps,
built from the reference sources) on this machine's host cores, one MPI rank per
core through the project's shared-memory MPI shim, on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SHAPE = (256, 256, 256)
WORKLOAD = ("spherical Riemann 256^3, FP64 Euler, WENO5-Z (reference :80 stencil), AUSM, "
            "outlet faces, TVD-RK3 CFL 0.5")

# Algorithmic FP64 operations per cell, counted from the reference's expressions
# (add/sub/mul/div/sqrt = 1, abs = 0, pow(x,2) = 1), per the cited reference lines.
FLOPS = {
    "con2prim": 46,        # src/physicsModel.cpp:315-353, :1000-1054
    "AUSM": 82,            # src/physicsModel.cpp:557-597 + RiemannAUSM :762-850, per direction
    "LF": 60,              # RiemannLF :940-979, per direction
    "AUSMp": 94,           # RiemannAUSMp :852-938, per direction
    "weno5js": 67,         # per face, variable and split: src/weno5js.cpp:75-108
    "weno5z": 74,          # src/weno5z.cpp:74-109
    "weno7js": 146,        # src/weno7js.cpp:84-136
    # compact schemes, per face, variable and split: the interior row (crweno5
    # src/crweno5.cpp:135-163: 68; hccs src/hccs.cpp:154-187: 104) + the Thomas solve
    # (src/crweno5.cpp:207-218: 10 per row)
    "crweno5": 78,
    "hccs": 114,
    "combine": 1,          # per face and variable: src/euler3d.cpp:45-49
    "cd6": 8,              # per cell and field: 3 differences, 3 products, 2 sums
                           # (src/centraldifference6th.cpp:26-43)
    "difference": 1,       # per cell and variable: src/euler3d.cpp:163-169
    "rhs_add": 1,          # per cell and variable: src/euler3d.cpp:405,419
    "rk": 14.0 / 3.0,      # per cell and variable, mean of stages 4,5,5: src/TVD-RK3.cpp:57-136
}
# HBM bytes a right-hand-side sweep (the launch profile_sweep times) cannot avoid per
# cell: Q (40) + jac (8) + its direction's metric (24), plus the RHS write (xi) or the
# RHS read and write (eta, zeta).
SWEEP_BYTES = {0: 72 + 40, 1: 72 + 80, 2: 72 + 80}
# DRAM bytes per cell the same launches moved under ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of a 192^3 block, whose every array is larger than L2, divided by
# its cells; a launch's traffic grows with its cells).
SWEEP_TRAFFIC = {0: 108.1, 1: 152.1, 2: 150.8}
# The same for the pipelined sweeps (pipe_sweep_kernel, tile 2 x 128, 192^3): their TMA
# boxes carry each tile's halo, so they read 10-14% more.
SWEEP_TRAFFIC_PIPE = {0: 118.7, 1: 164.0, 2: 158.9}


def sweep_flops_per_cell(d: int, scheme: str = "weno5z", riemann: str = "AUSM",
                         ns: bool = False) -> float:
    """Algorithmic flops per cell of one right-hand-side sweep along d (no RK update); ns:
    plus the direction's cd6 differences of the 4 viscous fluxes and their subtraction."""
    f = FLOPS[riemann] + 10 * FLOPS[scheme] + 5 * FLOPS["combine"] + 5 * FLOPS["difference"]
    if d == 0:
        f += FLOPS["con2prim"]
    else:
        f += 5 * FLOPS["rhs_add"]
    if ns:
        f += 4 * FLOPS["cd6"] + 4 * FLOPS["rhs_add"]
    return f


# ---------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.p = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if self.p is None or self.out is None:
            return None
        self.out.flush()
        rows = [r.split(",") for r in Path(self.out.name).read_text().splitlines() if r.strip()]
        os.unlink(self.out.name)
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "power_w_max": max(pw) if pw else None, "samples": len(rows)}


# ---------------------------------------------------------------------------------
# the reference on the host cores
# ---------------------------------------------------------------------------------
def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def decompose(shape, nranks):
    """Split shape into nranks = 2^k blocks by halving the largest extent."""
    parts = [1, 1, 1]
    n = nranks
    while n > 1:
        ext = [shape[d] // parts[d] for d in range(3)]
        d = int(np.argmax(ext))
        if ext[d] % 2 or (ext[d] // 2) % 4 or ext[d] // 2 < 12:
            break
        parts[d] *= 2
        n //= 2
    return parts


def reference_case(shape, nranks):
    """A refrun.Case of the workload split over nranks blocks (outlet outer faces)."""
    from oracle import refrun as R
    from nuc3d_b200 import cases as C
    parts = decompose(shape, nranks)
    nr = parts[0] * parts[1] * parts[2]
    bs = [shape[d] // parts[d] for d in range(3)]
    xs = [np.arange(shape[d] + 1, dtype=np.float64) / shape[d] for d in range(3)]
    rank_of = lambda a, b, c: a + parts[0] * (b + parts[1] * c)  # noqa: E731
    nodes, topo, q0 = [], [], []
    for c in range(parts[2]):
        for b in range(parts[1]):
            for a in range(parts[0]):
                lo = [a * bs[0], b * bs[1], c * bs[2]]
                sl = [slice(lo[d], lo[d] + bs[d] + 1) for d in range(3)]
                Z, Y, X = np.meshgrid(xs[2][sl[2]], xs[1][sl[1]], xs[0][sl[0]], indexing="ij")
                nodes.append((X, Y, Z))
                pos = [a, b, c]
                lines = []
                for f in range(6):
                    d, side = f // 2, f % 2
                    p2 = list(pos)
                    p2[d] += 1 if side else -1
                    if 0 <= p2[d] < parts[d]:
                        lines.append(f"{rank_of(*p2)} {f ^ 1}")
                    else:
                        lines.append("-1 1")
                topo.append(lines)
                h = [1.0 / shape[d] for d in range(3)]
                xc = [(lo[d] + np.arange(bs[d]) + 0.5) * h[d] for d in range(3)]
                Zc, Yc, Xc = np.meshgrid(xc[2], xc[1], xc[0], indexing="ij")
                prim = R.spherical_riemann_prim(Xc, Yc, Zc)
                jac = np.full(Xc.shape, 1.0 / (h[0] * h[1] * h[2]))
                q0.append(C.prim_to_q(prim, jac, 1.4))
    case = R.Case(model="Euler3d", riemann="AUSM", schemes=("weno5z",) * 3,
                  params={"Reynolds": 1000.0, "Mach": 1.0, "Pt": 0.72, "Gamma": 1.4,
                          "T_ref": 110.4, "T_inf": 288.0, "T_wall": 1.0},
                  nodes=nodes, bc_topo=topo, q0=q0, start_step=1)
    return case, nr


def run_reference(shape, steps, warmup, timeout=1800):
    """Reference block::solve time on the host cores: (Mcell-steps/s, cores, sample)."""
    from oracle import refrun as R
    cores = host_cores()
    nranks = 1
    while nranks * 2 <= min(cores, 256):
        nranks *= 2
    case, nr = reference_case(shape, nranks)
    out = R.run(case, "time", steps, warmup, timeout=timeout)[0]
    rec = json.loads(out.strip().splitlines()[-1])
    cells = shape[0] * shape[1] * shape[2]
    value = cells * steps / rec["solve_seconds"] / 1e6
    sample = (f"{steps} timed + {warmup} warm-up TVD-RK3 steps of the {shape[0]}x{shape[1]}x"
              f"{shape[2]} workload split into {nr} blocks, one reference rank (process) per core; "
              f"time = sum over steps of max over ranks of block::solve wall time")
    return value, nr, sample, rec["solve_seconds"]


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    shape = SHAPE
    cells = shape[0] * shape[1] * shape[2]
    # bound the run: ~0.15 Mcell-steps/s per core for this scheme on one core
    est = cells / (0.15e6 * max(1, min(host_cores(), 256))) * (args.steps + args.warmup)
    if est > 300.0:
        shape = (128, 128, 128)
        cells = shape[0] ** 3
    value, nr, sample, secs = run_reference(shape, args.steps, args.warmup)
    line = {
        "impl": "reference", "metric": "Mcell-RK3-steps/s", "value": value,
        "cpu_model": cpu_model(),
        "unit": "Mcell-RK3-steps/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": cells, "parallelism": f"{nr} MPI ranks on CPU"},
        "cpu_baseline": {"value": value, "unit": "Mcell-RK3-steps/s", "cores": nr,
                         "kind": "reference", "sample": sample, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "Mcell-RK3-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------
# multi-rank bookkeeping (replicas: one independent block per GPU, no data-path collective)
# ---------------------------------------------------------------------------------
def rank_max(x: float, dist=None, device="cpu") -> float:
    """The slowest rank's time: all-reduce(MAX) over the process group (identity alone)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, cells_per_rank: int, steps: int, ms_max: float) -> float:
    """Mcell-RK3-steps/s of the whole job: every rank's cells over the slowest rank's time."""
    return world * cells_per_rank * steps / (ms_max * 1e-3) / 1e6


# ---------------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------------
def ours(args):
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                    gamma=1.4, cfl=0.5, exact=args.exact, weno5z_compat=True)
    q0, _ = C.spherical_riemann(SHAPE)
    cells = int(np.prod(SHAPE))
    s = nb.Solver(cfg, device=local)
    b = s.add_block(*SHAPE, *C.outlet_faces())
    # metrics by block::getJacobians from the unit-box nodes on the GPU: the reference's own
    s.set_nodes(b, *C.unit_box_nodes(SHAPE))
    s.finalize()
    stream = torch.cuda.Stream(device=dev)
    s.set_stream(stream.cuda_stream)
    s.set_q(b, q0)
    # sweep tile shapes per direction, timed on this grid (outside every timed region);
    # --tiles pins them instead (profiler runs, whose timings would mislead the autotuner)
    if args.tiles:
        s.set_tiles(args.tiles)
        tiles = s.get_tiles()
        if args.pipe_mask is not None:
            s.set_pipeline(args.pipe_mask if args.pipe_mask > 1 else bool(args.pipe_mask))
    else:
        tiles = s.autotune(reps=3)["shape"]
    pipe_dirs_step = s.pipeline()  # directions the timed steps run pipelined (bit d)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        s.sync()

    def max_over_ranks(x):
        return rank_max(x, dist, dev)

    # ---- device-resident timing ----
    s.step(args.warmup)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            s.step(args.steps, sync=False)
            ev1.record(stream)
        ev1.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    s.sync()
    status = s.status()
    resets = s.energy_resets()  # over the warm-up and timed steps
    value = whole_job_rate(world, cells, args.steps, ms)

    # ---- end to end through the public API with pinned host buffers ----
    # nuc3d_solve_host: block::solve on host arrays, every step uploads Q from the host
    # array and writes the new Q back there (the download of a step and the upload of the
    # next share the PCIe link in both directions, chunk by chunk)
    host_q = torch.empty(5 * cells, dtype=torch.float64, pin_memory=True)
    host_q.numpy()[:] = s.get_q(b).reshape(-1)
    e2e_steps = max(3, min(args.steps, 10))
    s.solve_host([host_q.data_ptr()], 2)  # warm-up of the copy path
    barrier()
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    s.solve_host([host_q.data_ptr()], e2e_steps)
    ev3.record(stream)
    ev3.synchronize()
    e2e_ms = max_over_ranks(ev2.elapsed_time(ev3))
    e2e_value = whole_job_rate(world, cells, e2e_steps, e2e_ms)
    # the same copies issued one after the other (upload, step, download, wait)
    s.set_q_ptr(b, host_q.data_ptr())
    s.step(1, sync=False)
    s.get_q_ptr(b, host_q.data_ptr())
    ev4, ev5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev4.record(stream)
    for _ in range(e2e_steps):
        s.set_q_ptr(b, host_q.data_ptr())
        s.step(1, sync=False)
        s.get_q_ptr(b, host_q.data_ptr())
    ev5.record(stream)
    ev5.synchronize()
    e2e_serial_value = whole_job_rate(world, cells, e2e_steps, max_over_ranks(ev4.elapsed_time(ev5)))

    # ---- hybrid WENO-Z with the learned face sensor: same workload, same step count ----
    hybrid = None
    if not args.exact:
        from nuc3d_b200 import sensor as SENS
        warm = 2
        s.set_q(b, q0)
        s.step(warm + args.steps)
        rho_plain = s.get_q(b)[0]
        s.set_q(b, q0)
        s.set_sensor(SENS.load_weights(), SENS.DEFAULT_THRESHOLD)
        htiles = s.get_tiles() if args.tiles else s.autotune(reps=3)["shape"]
        s.step(warm)  # includes the capture of the hybrid step graph
        barrier()
        ev4, ev5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev4.record(stream)
        s.step(args.steps, sync=False)
        ev5.record(stream)
        ev5.synchronize()
        s.sync()
        hms = max_over_ranks(ev4.elapsed_time(ev5))
        rho_h = s.get_q(b)[0]
        s.set_sensor(None)
        # the plain grid's shapes and pipelined directions again (the hybrid's autotune set
        # its own; the plain choice comes back from the autotuner's cache without timing)
        if args.tiles:
            s.set_tiles(tiles)
            if args.pipe_mask is not None:
                s.set_pipeline(args.pipe_mask if args.pipe_mask > 1 else bool(args.pipe_mask))
        else:
            s.autotune(reps=3)
        hv = whole_job_rate(world, cells, args.steps, hms)
        hybrid = {"value": hv, "unit": "Mcell-RK3-steps/s", "ms_per_step": hms / args.steps,
                  "vs_plain": hv / value, "logit_threshold": SENS.DEFAULT_THRESHOLD,
                  "l1_density_error_vs_plain": float(np.abs(rho_h - rho_plain).sum() /
                                                     np.abs(rho_plain).sum()),
                  "steps_compared": warm + args.steps, "tile_shapes": list(htiles)}

    # ---- roofline of the dominant kernel ----
    s.set_q(b, q0)
    per = {d: s.profile_sweep(d, reps=5) for d in range(3)}
    pipelined = s.pipeline()
    if pipelined:  # the same launches with one tile per CTA, for comparison
        s.set_pipeline(False)
        per_plain = {d: s.profile_sweep(d, reps=5) for d in range(3)}
        s.set_pipeline(True)
    else:
        per_plain = None
    dom = max(per, key=per.get)
    flops = sweep_flops_per_cell(dom) * cells
    achieved = flops / (per[dom] * 1e-3) / 1e12
    peak = nb.fp64_peak_tflops(local)
    hbm_achieved = SWEEP_BYTES[dom] * cells / (per[dom] * 1e-3) / 1e9
    try:
        hbm_peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
        hbm_src = "MEASURED_PEAKS.json"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback"

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        s.close()
        return 0

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            # block::solve timed over 10 steps after 2 warm-up steps
            v, nr, sample, _ = run_reference(SHAPE, 10, 2)
            cpu = {"value": v, "unit": "Mcell-RK3-steps/s", "cores": nr, "kind": "reference",
                   "sample": sample, "cpu_model": cpu_model()}
        except Exception as e:  # the baseline is a report, never a reason to fail the bench
            cpu = {"value": None, "unit": "Mcell-RK3-steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}".splitlines()[0][:200], "cpu_model": cpu_model()}
    # the batched multi-block Navier-Stokes workload (24 uneven blocks) and the
    # shock-turbulence workload (plain against the learned hybrid), on this GPU
    launches = s.kernels_per_step() * args.steps
    turb = shock = bl = compact = None
    if world == 1 and not args.no_turbulence:
        s.close()
        try:
            turb = turbulence24(args, with_cpu=not args.no_cpu_baseline)
        except Exception as e:  # reported, never a reason to fail the bench
            turb = {"unavailable": f"{type(e).__name__}: {e}".splitlines()[0][:300]}
        try:
            shock = shock_turbulence(args)
        except Exception as e:
            shock = {"unavailable": f"{type(e).__name__}: {e}".splitlines()[0][:300]}
        try:
            bl = boundary_layer(args)
        except Exception as e:
            bl = {"unavailable": f"{type(e).__name__}: {e}".splitlines()[0][:300]}
        try:
            compact = compact256(args)
        except Exception as e:
            compact = {"unavailable": f"{type(e).__name__}: {e}".splitlines()[0][:300]}

    line = {
        "metric": "Mcell-RK3-steps/s", "value": value, "unit": "Mcell-RK3-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells_per_gpu": cells,
                   "arith": "reference-order (no FMA)" if args.exact else "fast (FMA, 1 div/face)",
                   "l2": "no flush: 3 state buffers of 671 MB + RHS + metrics = 4 GB > 126 MB L2",
                   "parallelism": f"replicas x{world} (one independent block per GPU)",
                   "tile_shapes": list(tiles),
                   "pipelined_dirs": pipe_dirs_step,
                   "status_bits": status,
                   "energy_reset_cells": resets,
                   "energy_reset_note": "cells whose energy con2prim reset (e < 0, "
                                        "src/physicsModel.cpp:324-332), once per cell and "
                                        "right-hand side, over the warm-up and timed steps",
                   "metrics": "block::getJacobians of the unit-box nodes (the reference's)"},
        "clocks": clk.summary(),
        "e2e": {"value": e2e_value, "unit": "Mcell-RK3-steps/s",
                "h2d_bytes_per_step": 5 * cells * 8, "d2h_bytes_per_step": 5 * cells * 8,
                "steps": e2e_steps, "api": "nuc3d_solve_host (host Q in place, every step)",
                "serial_copies_value": e2e_serial_value},
        "gpu_launches": launches,
        "roofline": {
            "bound": "fp64",
            "kernel": (f"{'pipe_sweep_kernel' if (pipelined >> dom) & 1 else 'sweep_kernel'}<{dom}> "
                       f"({'xi eta zeta'.split()[dom]}, right-hand side)"),
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "measured live: libnuc3d_probe DFMA microbenchmark",
            "flops_per_cell": sweep_flops_per_cell(dom), "ms_per_launch": per[dom],
            "ms_per_launch_all": per,
            "pipelined": bool((pipelined >> dom) & 1),
            "pipelined_dirs": pipelined,
            "ms_per_launch_one_tile_per_cta": per_plain,
            "traffic": ((SWEEP_TRAFFIC_PIPE if (pipelined >> dom) & 1 else SWEEP_TRAFFIC)[dom] * cells),
            "traffic_unit": "bytes per launch",
            "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": hbm_achieved / hbm_peak, "peak_source": hbm_src,
                    "bytes_per_cell": SWEEP_BYTES[dom]},
        },
        "cpu_baseline": cpu,
        "hybrid": hybrid,
        "turbulence24": turb,
        "shock_turbulence": shock,
        "boundary_layer": bl,
        "compact": compact,
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if turb is None:
        s.close()
    return 0


SHOCK_WORKLOAD = ("Mach 1.5 normal shock at x = pi/2 in decaying isotropic turbulence (the 24-block "
                  "case's spectrum, Mt 0.6, Re_lambda 100), 512x256x256 FP64 Navier-Stokes, inflow "
                  "x-, outflow x+, periodic y/z, WENO5-Z, AUSM, cd6, TVD-RK3 CFL 0.5")


def shock_turbulence(args, steps=10, warm=2):
    """Plain WENO-Z against the hybrid with the learned face sensor (trained on the
    Taylor-Green and spherical-blast runs only, so this flow is held out) on the
    shock-turbulence workload: Mcell-RK3-steps/s of both from the same state over the same
    steps, the L1 density error of the hybrid against plain, and the shock position."""
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    from nuc3d_b200 import sensor as SENS
    shape = (512, 256, 256)
    prim, re, inlet, nodes = C.shock_turbulence(shape)
    h = 2.0 * math.pi / shape[1]
    q0 = C.prim_to_q(prim, np.full(prim.shape[1:], 1.0 / (h * h * h)), 1.4)
    del prim
    cells = int(np.prod(shape))
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                            reynolds=re, mach=0.6, cfl=0.5, exact=False))
    t, i = C.shock_faces()
    vals = np.zeros((6, 5))
    vals[0] = inlet
    b = s.add_block(*shape, t, i, vals)
    s.set_nodes(b, *nodes)
    del nodes
    s.finalize()
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)

    def run(label):
        s.set_q(b, q0)
        s.set_time(0.0)
        tiles = s.autotune(reps=2)["shape"]
        s.set_q(b, q0)
        s.step(warm)
        s.sync()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.step(steps, sync=False)
        ev1.record(stream)
        ev1.synchronize()
        s.sync()
        ms = ev0.elapsed_time(ev1) / steps
        rho = s.get_q(b)[0] * (1.0 / (h * h * h))  # U/J -> rho on the uniform mesh
        return ms, rho, {"tile_shapes": list(tiles), "pipelined_dirs": s.pipeline()}

    ms_p, rho_p, tiles_p = run("plain")
    s.set_sensor(SENS.load_weights(), SENS.DEFAULT_THRESHOLD)
    ms_h, rho_h, tiles_h = run("hybrid")
    # the same hybrid deciding by hccs's hand-made theta switch instead of the network
    theta = []
    for tmin in (0.5, 0.9):
        s.set_sensor_theta(tmin)
        ms_t, rho_t, tiles_t = run("theta")
        theta.append({"theta_min": tmin, "value": cells / (ms_t * 1e-3) / 1e6, "ms_per_step": ms_t,
                      "vs_plain": ms_p / ms_t, **tiles_t,
                      "l1_density_error_vs_plain": float(np.abs(rho_t - rho_p).sum() / np.abs(rho_p).sum()),
                      "shock_x": C.shock_position(rho_t, h)})
        del rho_t
    s.set_sensor(None)
    s.close()
    vp = cells / (ms_p * 1e-3) / 1e6
    vh = cells / (ms_h * 1e-3) / 1e6
    return {"workload": SHOCK_WORKLOAD, "cells": cells, "steps_compared": warm + steps,
            "plain": {"value": vp, "unit": "Mcell-RK3-steps/s", "ms_per_step": ms_p,
                      **tiles_p},
            "hybrid": {"value": vh, "unit": "Mcell-RK3-steps/s", "ms_per_step": ms_h,
                       **tiles_h, "logit_threshold": SENS.DEFAULT_THRESHOLD},
            "vs_plain": vh / vp,
            "l1_density_error_vs_plain": float(np.abs(rho_h - rho_p).sum() / np.abs(rho_p).sum()),
            "shock_x": {"initial": 0.5 * math.pi, "plain": C.shock_position(rho_p, h),
                        "hybrid": C.shock_position(rho_h, h)},
            "theta_switch": theta,
            "theta_switch_rule": "linear weights where the smallest hccs theta "
                                 "(src/hccs.cpp:177-181) of the face's density and pressure "
                                 "stencils, both splits, is at least theta_min",
            "sensor_training": "Taylor-Green vortex and spherical blast runs only (held out here)"}


COMPACT_WORKLOAD = ("smooth isentropic pressure pulse 256^3 (rho = 1 + 0.5 exp(-r^2/0.08^2), "
                    "p = rho^1.4/1.4, at rest), periodic faces, FP64 Euler, {scheme} in every "
                    "direction, AUSM, TVD-RK3 CFL 0.2 (at CFL 0.5 the reference's compact schemes "
                    "diverge on this pulse: NaN within 60 steps at 32^3, the reference itself)")


def compact256(args, steps=10, warm=3):
    """The compact schemes (crweno5, hccs) in every direction on a 256^3 Euler block: the
    throughput build's fused line sweep (compact_line_kernel, one kernel per direction)
    against its three-kernel path (rows to HBM, Thomas per system, faces), step times and
    the fused sweep's per-launch roofline."""
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C

    torch.cuda.set_device(0)
    q0, _ = C.gaussian_pulse(SHAPE)
    cells = int(np.prod(SHAPE))
    stream = torch.cuda.Stream()
    peak = nb.fp64_peak_tflops(0)
    out = {}
    for scheme in ("crweno5", "hccs"):
        # CFL 0.2: at 0.5 the reference's crweno5 and hccs diverge on this pulse within
        # 60 steps (NaN at 32^3, run on the reference itself), the same with periodic or
        # outlet faces and with LF or AUSM splitting; the blast's discontinuity drives them
        # to negative pressure at any CFL
        s = nb.Solver(nb.Config(scheme_ivs=(scheme,) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                                cfl=0.2, exact=False))
        b = s.add_block(*SHAPE, *C.periodic_faces())
        s.set_nodes(b, *C.unit_box_nodes(SHAPE))
        s.finalize()
        s.set_stream(stream.cuda_stream)
        res = {}
        for fused in (True, False):
            s.set_compact_solver(fused)
            s.set_q(b, q0)
            s.set_time(0.0)
            s.step(warm)
            s.sync()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with ClockSampler(0) as clk:
                ev0.record(stream)
                s.step(steps, sync=False)
                ev1.record(stream)
                ev1.synchronize()
            s.sync()
            ms = ev0.elapsed_time(ev1) / steps
            per = [s.profile_sweep(d, reps=3) for d in range(3)]
            res[fused] = {"value": cells / (ms * 1e-3) / 1e6, "ms_per_step": ms,
                          "sweep_ms_per_launch": per, "kernels_per_step": s.kernels_per_step(),
                          "clocks": clk.summary()}
        s.close()
        per = res[True]["sweep_ms_per_launch"]
        dom = int(np.argmax(per))
        f = sweep_flops_per_cell(dom, scheme=scheme)
        achieved = f * cells / (per[dom] * 1e-3) / 1e12
        out[scheme] = {
            "workload": COMPACT_WORKLOAD.format(scheme=scheme), "unit": "Mcell-RK3-steps/s",
            "fused": res[True], "three_kernels": res[False],
            "vs_three_kernels": res[True]["value"] / res[False]["value"],
            "roofline": {"bound": "fp64", "kernel": f"compact_line_kernel<{dom}> "
                         f"({'xi eta zeta'.split()[dom]})", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak, "flops_per_cell": f,
                         "peak_source": "measured live: libnuc3d_probe DFMA microbenchmark",
                         "ms_per_launch": per[dom]}}
    return out


BL_WORKLOAD = ("supersonic flat-plate boundary layer, Ma 2.25, Re_x 1e5 at the inflow (Re_delta "
               "1581), isothermal wall T_w/T_inf 1.9, Gaussian bump h 0.5 delta w 2 delta, "
               "1024x256x128 cells on a tanh wall-normal stretched mesh in 4x2x2 = 16 uneven "
               "blocks; inlet x-, outlet x+, wall y-, outlet y+, periodic z; FP64 Navier-Stokes, "
               "WENO5-Z, AUSM, cd6, TVD-RK3 CFL 0.5")


def _bl_compare(shape, steps, warm, thresholds, autotune=True):
    """Plain WENO-Z, the hybrid at each logit threshold and plain WENO5-JS on the
    boundary-layer grid of `shape`, all from the same state over warm + steps steps: device
    ms per step and, per variant, the volume-weighted L1 density distance from plain
    WENO-Z (U/J = rho x cell volume, so the L1 norm of U/J is that of rho weighted by
    volume)."""
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    from nuc3d_b200 import sensor as SENS

    blocks, types, ids, values, prm = C.boundary_layer(shape)
    stream = torch.cuda.Stream()

    def solver(scheme):
        s = nb.Solver(nb.Config(scheme_ivs=(scheme,) * 3, riemann="AUSM", model="NavierStokes3d",
                                reynolds=prm["Reynolds"], mach=prm["Mach"], t_wall=prm["T_wall"],
                                cfl=0.5, exact=False))
        for r, b in enumerate(blocks):
            s.add_block(*b["shape"], types[r], ids[r], values[r])
        for r, b in enumerate(blocks):
            s.set_nodes(r, *b["nodes"])
        s.finalize()
        s.set_stream(stream.cuda_stream)
        if "q" not in blocks[0]:
            for r, b in enumerate(blocks):
                b["q"] = np.ascontiguousarray(C.prim_to_q(b["prim"], s.get_metrics(r)["jac"],
                                                          prm["Gamma"]))
                del b["prim"]
        return s

    def run(s):
        tiles = None
        if autotune:
            for r, b in enumerate(blocks):
                s.set_q(r, b["q"])
            s.set_time(0.0)
            tiles = list(s.autotune(reps=2)["shape"])
        for r, b in enumerate(blocks):
            s.set_q(r, b["q"])
        s.set_time(0.0)
        s.step(warm)
        s.sync()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        s.step(steps, sync=False)
        ev1.record(stream)
        ev1.synchronize()
        s.sync()
        mass = np.concatenate([s.get_q(r)[0].ravel() for r in range(len(blocks))])
        return {"ms_per_step": ev0.elapsed_time(ev1) / steps, "tile_shapes": tiles,
                "pipelined_dirs": s.pipeline(), "status_bits": s.status(),
                "time": s.time_dt()[0]}, mass

    s = solver("weno5z")
    plain, m_p = run(s)
    l1 = lambda m: float(np.abs(m - m_p).sum() / np.abs(m_p).sum())  # noqa: E731
    hyb = []
    for th in thresholds:
        s.set_sensor(SENS.load_weights(), th)
        h, m_h = run(s)
        h.update(logit_threshold=th, vs_plain=plain["ms_per_step"] / h["ms_per_step"],
                 l1_density_error_vs_plain=l1(m_h))
        hyb.append(h)
        del m_h
    s.set_sensor(None)
    s.close()
    s = solver("weno5js")
    js, m_js = run(s)
    s.close()
    js["l1_density_distance_vs_plain"] = l1(m_js)
    return {"cells": int(np.prod(shape)), "blocks": len(blocks),
            "block_shapes": [list(b["shape"]) for b in blocks], "steps": warm + steps,
            "plain": plain, "hybrid": hyb, "weno5js": js}


def boundary_layer(args, thresholds=(-4.0, -2.0, 0.0)):
    """The boundary-layer workload on one GPU: the 16 blocks in one context (on-device ghost
    copies, one launch per sweep over all blocks), metrics from the nodes on the device.
    Throughput of plain WENO-Z and of the learned hybrid (batched over the same blocks) at
    each logit threshold on the full 1024 x 256 x 128 grid over 12 steps.  Their accuracy
    over a horizon in which the flow over the bump develops (800 steps; the line gives the
    time reached, in delta / U_inf) on the same case at 256 x 64 x 32: the volume-weighted L1 density
    distance of each hybrid from plain WENO-Z, matched against the distance between two
    plain fifth-order schemes (WENO5-JS and WENO5-Z); a hybrid within it changes the
    solution less than the choice of WENO weights does."""
    full = _bl_compare((1024, 256, 128), 10, 2, thresholds)
    small = _bl_compare((256, 64, 32), 790, 10, thresholds, autotune=False)
    target = small["weno5js"]["l1_density_distance_vs_plain"]
    ok = [k for k, h in enumerate(small["hybrid"]) if h["l1_density_error_vs_plain"] <= target]
    best = max(ok, key=lambda k: full["hybrid"][k]["vs_plain"]) if ok else None
    cells = full["cells"]
    pv = cells / (full["plain"]["ms_per_step"] * 1e-3) / 1e6
    return {"workload": BL_WORKLOAD, "cells": cells, "blocks": full["blocks"],
            "block_shapes": full["block_shapes"], "steps_timed": 10,
            "plain": dict(full["plain"], value=pv, unit="Mcell-RK3-steps/s"),
            "hybrid": [dict(h, value=cells / (h["ms_per_step"] * 1e-3) / 1e6,
                            l1_density_error_vs_plain_800_steps=small["hybrid"][k]["l1_density_error_vs_plain"])
                       for k, h in enumerate(full["hybrid"])],
            "weno5js": full["weno5js"],
            "matched_error": {
                "grid": "the same case at 256x64x32 cells (16 blocks), 800 steps, t = %.3g" % small["plain"]["time"],
                "target_l1": target,
                "target": "L1 density distance of plain WENO5-JS from plain WENO5-Z",
                "hybrid_l1": [h["l1_density_error_vs_plain"] for h in small["hybrid"]],
                "hybrid_at_target": ({"logit_threshold": thresholds[best],
                                      "vs_plain": full["hybrid"][best]["vs_plain"]}
                                     if best is not None else None)},
            "sensor_training": "Taylor-Green vortex and spherical blast runs only (held out here)",
            "metrics": "nuc3d_block_set_nodes (block::getJacobians on the device)"}


TURB_WORKLOAD = ("decaying isotropic turbulence, 2pi periodic box in 24 uneven blocks (per-axis "
                 "sizes from {48,64,96,128,160}, seed 99), 40.1M cells, FP64 Navier-Stokes, "
                 "WENO5-Z, AUSM, cd6, Mt 0.6, Re_lambda 100, TVD-RK3 CFL 0.5")


def turbulence24_reference(seed_parts=99, sizes=(16, 24, 32, 48), steps=3, warmup=1):
    """The reference on the host cores for the 24-block workload: the same 2 x 3 x 4
    periodic tensor-product partition, physics and schemes, block sizes drawn from `sizes`
    (the full 40 M cells would need its mesh written and parsed as text, minutes of I/O),
    one reference rank (process) per block."""
    from oracle import refrun as R
    from nuc3d_b200 import cases as C
    from nuc3d_b200.metrics import metrics_from_nodes
    parts = C.uneven_blocks(sizes=sizes, seed=seed_parts)
    n = [sum(p) for p in parts]
    x, y, z = R.box_nodes(*n, hi=(2.0 * math.pi,) * 3)
    prim, re = C.isotropic_turbulence(tuple(n), seed=7)
    types, ids = C.block_topology(parts)
    off = [np.concatenate([[0], np.cumsum(p)]) for p in parts]
    nodes, q0 = [], []
    for c in range(len(parts[2])):
        for b in range(len(parts[1])):
            for a in range(len(parts[0])):
                lo = (off[0][a], off[1][b], off[2][c])
                hi = (off[0][a + 1], off[1][b + 1], off[2][c + 1])
                nsl = tuple(slice(lo[d], hi[d] + 1) for d in (2, 1, 0))
                csl = tuple(slice(lo[d], hi[d]) for d in (2, 1, 0))
                xyz = tuple(arr[nsl] for arr in (x, y, z))
                m = metrics_from_nodes(*xyz)
                nodes.append(xyz)
                q0.append(np.ascontiguousarray(C.prim_to_q(prim[(slice(None),) + csl], m["jac"], 1.4)))
    topo = [[f"{types[r][f]} {ids[r][f]}" for f in range(6)] for r in range(len(nodes))]
    case = R.Case(model="NavierStokes3d", riemann="AUSM", schemes=("weno5z",) * 3,
                  params={"Reynolds": re, "Mach": 0.6, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
                          "T_inf": 288.0, "T_wall": 1.0},
                  nodes=nodes, bc_topo=topo, q0=q0, start_step=1)
    out = R.run(case, "time", steps, warmup, timeout=1800)[0]
    rec = json.loads(out.strip().splitlines()[-1])
    cells = int(np.prod(n))
    value = cells * steps / rec["solve_seconds"] / 1e6
    sample = (f"{steps} timed + {warmup} warm-up steps of the 24-block partition with block sizes "
              f"from {list(sizes)} ({cells} cells), one reference rank (process) per block on "
              f"{host_cores()} host cores")
    return {"value": value, "unit": "Mcell-RK3-steps/s", "cores": min(len(nodes), host_cores()),
            "kind": "reference", "sample": sample, "cpu_model": cpu_model()}


def turbulence24(args, with_cpu=False):
    """The batched multi-block Navier-Stokes workload on one GPU: every block of the grid in
    one context (on-device ghost copies), one launch per sweep over all blocks, the step a
    CUDA graph, tile shapes from nuc3d_autotune.  Returns its bench line (a dict)."""
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C

    torch.cuda.set_device(0)
    parts = C.uneven_blocks(seed=99)
    n = [sum(p) for p in parts]
    prim, re = C.isotropic_turbulence(tuple(n), seed=7)
    types, ids = C.block_topology(parts)
    off = [np.concatenate([[0], np.cumsum(p)]) for p in parts]
    h = [2 * math.pi / n[d] for d in range(3)]
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                            reynolds=re, mach=0.6, cfl=0.5, exact=args.exact))
    boxes = [((a, b, c), (parts[0][a], parts[1][b], parts[2][c]))
             for c in range(len(parts[2])) for b in range(len(parts[1])) for a in range(len(parts[0]))]
    for r, (_, sh) in enumerate(boxes):
        s.add_block(*sh, types[r], ids[r])
    mets = [C.uniform_metrics(sh, lo=(0, 0, 0), hi=tuple(h[d] * sh[d] for d in range(3)))
            for _, sh in boxes]
    for r, m in enumerate(mets):
        s.set_metrics(r, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    qs = []
    for r, ((a, b, c), sh) in enumerate(boxes):
        sl = (slice(None), slice(off[2][c], off[2][c + 1]), slice(off[1][b], off[1][b + 1]),
              slice(off[0][a], off[0][a + 1]))
        qs.append(np.ascontiguousarray(C.prim_to_q(prim[sl], mets[r]["jac"], 1.4)))
        s.set_q(r, qs[r])
    cells = int(np.prod(n))
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    if args.tiles:
        s.set_tiles(args.tiles)
        tiles = s.get_tiles()
    else:
        tiles = s.autotune(reps=2)["shape"]
    s.step(args.warmup)
    s.sync()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        ev0.record(stream)
        s.step(args.steps, sync=False)
        ev1.record(stream)
        ev1.synchronize()
    s.sync()
    ms = ev0.elapsed_time(ev1)
    # end to end: every block's Q from pinned host arrays and back, every step
    host = [torch.empty(q.size, dtype=torch.float64, pin_memory=True) for q in qs]
    for hq, q in zip(host, qs):
        hq.numpy()[:] = q.reshape(-1)
    e2e_steps = max(3, min(args.steps, 10))
    s.solve_host([hq.data_ptr() for hq in host], 1)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    s.solve_host([hq.data_ptr() for hq in host], e2e_steps)
    ev3.record(stream)
    ev3.synchronize()
    e2e_ms = ev2.elapsed_time(ev3)
    per = [s.profile_sweep(d, reps=3) for d in range(3)]
    dom = int(np.argmax(per))
    flops = sweep_flops_per_cell(dom, ns=True) * cells
    achieved = flops / (per[dom] * 1e-3) / 1e12
    peak = nb.fp64_peak_tflops(0)
    cpu = None
    if with_cpu:
        try:
            cpu = turbulence24_reference()
        except Exception as e:
            cpu = {"value": None, "unit": "Mcell-RK3-steps/s", "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {e}".splitlines()[0][:200]}
    line = {
        "metric": "Mcell-RK3-steps/s", "value": whole_job_rate(1, cells, args.steps, ms),
        "unit": "Mcell-RK3-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": TURB_WORKLOAD, "cells_per_gpu": cells, "blocks": len(boxes),
                   "tile_shapes": list(tiles), "pipelined_dirs": s.pipeline(), "status_bits": s.status(),
                   "l2": "no flush: 40.1M cells x 5 doubles = 1.6 GB per state buffer > 126 MB L2"},
        "clocks": clk.summary(),
        "e2e": {"value": whole_job_rate(1, cells, e2e_steps, e2e_ms), "unit": "Mcell-RK3-steps/s",
                "h2d_bytes_per_step": 5 * cells * 8, "d2h_bytes_per_step": 5 * cells * 8,
                "steps": e2e_steps, "api": "nuc3d_solve_host (24 host arrays in place, every step)"},
        "gpu_launches": s.kernels_per_step() * args.steps,
        "sweep_ms_per_launch": per,
        "roofline": {"bound": "fp64",
                     "kernel": (f"{'pipe_sweep_kernel' if (s.pipeline() >> dom) & 1 else 'sweep_kernel'}"
                                f"<{dom}> ({'xi eta zeta'.split()[dom]}, NS)"),
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": "measured live: libnuc3d_probe DFMA microbenchmark",
                     "flops_per_cell": sweep_flops_per_cell(dom, ns=True),
                     "ms_per_launch": per[dom], "traffic": None},
        "cpu_baseline": cpu,
    }
    s.close()
    return line


def profile_case(args):
    """--profile-case: the workload at a chosen size, untimed -- the command ncu captures.
    Euler: the spherical Riemann problem (this file's workload); --ns: the Navier-Stokes
    Taylor-Green vortex (WENO5-JS, LF, periodic); --scheme S: S in every direction on the
    periodic smooth pulse (the compact key's workload).  --sweeps R launches each direction's
    right-hand-side sweep 1 + R times (the launches the roofline times) instead of stepping;
    --hybrid sets the learned face sensor."""
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    shape = (args.shape,) * 3
    if args.ns:
        cfg = nb.Config(scheme_ivs=("weno5js",) * 3, riemann="LF", model="NavierStokes3d",
                        mach=0.1, reynolds=1600.0, exact=args.exact)
        q, m = C.taylor_green(shape)
        faces = C.periodic_faces()
    elif args.scheme:
        # the compact bench key's workload: the periodic smooth pulse at CFL 0.2
        cfg = nb.Config(scheme_ivs=(args.scheme,) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                        cfl=0.2, exact=args.exact)
        q, m = C.gaussian_pulse(shape)
        faces = C.periodic_faces()
    else:
        cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                        exact=args.exact, weno5z_compat=True)
        q, m = C.spherical_riemann(shape)
        faces = C.outlet_faces()
    s = nb.Solver(cfg)
    b = s.add_block(*shape, *faces)
    s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, q)
    if args.tiles:
        s.set_tiles(args.tiles)
    if args.hybrid:
        from nuc3d_b200 import sensor
        s.set_sensor(sensor.load_weights(), sensor.DEFAULT_THRESHOLD)
    if args.sweeps > 0:
        print([s.profile_sweep(d, args.sweeps) for d in range(3)])
    else:
        s.step(args.steps)
        t, dt = s.time_dt()
        print(f"{shape} steps={args.steps} time={t:.6g} dt={dt:.6g} status={s.status()}")
    s.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--exact", action="store_true", help="reference-order arithmetic")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-turbulence", action="store_true",
                    help="leave out the 24-block Navier-Stokes line of the default run")
    ap.add_argument("--tiles", type=lambda x: tuple(int(v) for v in x.split(",")), default=None,
                    help="sweep tile shapes per direction, e.g. 2,0,0 (default: nuc3d_autotune)")
    ap.add_argument("--pipe-mask", type=int, default=None,
                    help="with --tiles: pipelined directions, bit d = direction d (e.g. 4: zeta)")
    ap.add_argument("--workload", default="sphere256",
                    choices=["sphere256", "turbulence24", "shock_turbulence", "boundary_layer",
                             "compact"],
                    help="turbulence24: the 24-block Navier-Stokes grid on one GPU; "
                         "shock_turbulence / boundary_layer: plain against hybrid on those "
                         "grids (our arm only)")
    ap.add_argument("--profile-case", action="store_true",
                    help="untimed run of the workload at --shape (the target of ncu captures)")
    ap.add_argument("--shape", type=int, default=128, help="--profile-case: cells per axis")
    ap.add_argument("--sweeps", type=int, default=0, help="--profile-case: sweep launches")
    ap.add_argument("--ns", action="store_true", help="--profile-case: NS Taylor-Green")
    ap.add_argument("--hybrid", action="store_true", help="--profile-case: learned sensor")
    ap.add_argument("--scheme", default=None,
                    help="--profile-case: this scheme in every direction on the smooth pulse "
                         "(the compact key's workload)")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case(args)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload in ("shock_turbulence", "boundary_layer", "compact"):
        if args.impl == "reference" or args.gpus > 1:
            print(json.dumps({"impl": args.impl,
                              "unavailable": f"{args.workload} runs our arm on one GPU only"}))
            return 0
        fn = {"shock_turbulence": shock_turbulence, "boundary_layer": boundary_layer,
              "compact": compact256}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return 0
    if args.workload == "turbulence24":
        if args.impl == "reference" or args.gpus > 1:
            print(json.dumps({"impl": args.impl, "unavailable": "turbulence24 runs our arm on one GPU only"}))
            return 0
        print(json.dumps(turbulence24(args, with_cpu=not args.no_cpu_baseline)), flush=True)
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
