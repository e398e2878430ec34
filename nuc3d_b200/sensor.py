"""Learned face sensor for the hybrid WENO-Z path: data, training, weights.

    python -m nuc3d_b200.sensor train [--out PATH] [--seed S]

Faces and labels come from plain WENO-Z runs (nuc3d_sensor_record): the Taylor-Green
vortex (Navier-Stokes, Lax-Friedrichs) and the spherical Riemann problem (Euler, AUSM),
recorded every few steps in all three directions.  The network (19 -> 32 -> 32 -> 1,
ReLU) is trained with the library's CUDA kernels (nuc3d_sensor_loss_grad: forward with
BF16 rounding as in the tensor-core inference, BCE loss, backward; nuc3d_sensor_adam).
Torch supplies device buffers and the random permutation only.
"""
from __future__ import annotations

import argparse
import ctypes
import math
import sys
from pathlib import Path

import numpy as np

from . import Config, Solver, load_library
from . import cases as C

N_IN, N_HID = 19, 32
N_PARAMS = N_HID * N_IN + N_HID + N_HID * N_HID + N_HID + N_HID + 1
WEIGHTS = Path(__file__).resolve().parent / "sensor_weights.npy"
# Logit below which a face takes the linear weights: on the spherical Riemann problem the
# L1 density error against plain WENO-Z stays below 1e-3 (64^3 after 60 steps: 3.9e-4;
# 128^3 after 120: 8.2e-5), with about 40% of the training faces sent to linear weights.
DEFAULT_THRESHOLD = -4.0


def _torch():
    import torch
    return torch


def record(solver: Solver, dirs=(0, 1, 2), cap: int = 1 << 22):
    """Features (n, 19) float32, labels (n,) uint8 and face-grid positions of the current
    state, as CUDA tensors (concatenated over dirs) plus the per-direction counts."""
    torch = _torch()
    feats, labels, wheres, counts = [], [], [], []
    for d in dirs:
        f = torch.empty((cap, N_IN), dtype=torch.float32, device="cuda")
        y = torch.empty(cap, dtype=torch.uint8, device="cuda")
        w = torch.empty(cap, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        n = solver.sensor_record(d, f.data_ptr(), y.data_ptr(), w.data_ptr(), cap)
        feats.append(f[:n]); labels.append(y[:n]); wheres.append(w[:n]); counts.append(n)
    return torch.cat(feats), torch.cat(labels), torch.cat(wheres), counts


def _solver_tgv(n, exact=False):
    q, m = C.taylor_green((n, n, n))
    s = Solver(Config(scheme_ivs=("weno5z",) * 3, riemann="LF", model="NavierStokes3d",
                      reynolds=1600.0, mach=0.1, exact=exact))
    b = s.add_block(n, n, n, *C.periodic_faces())
    s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, q)
    return s


def _solver_sphere(n, exact=False):
    q, m = C.spherical_riemann((n, n, n))
    s = Solver(Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                      exact=exact))
    b = s.add_block(n, n, n, *C.outlet_faces())
    s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, q)
    return s


def dataset(n=64, snapshots=(0, 20, 60, 120), seed=0, max_faces=1 << 22):
    """Training faces from the two plain runs; returns CUDA tensors (x, y)."""
    torch = _torch()
    xs, ys = [], []
    for make in (_solver_tgv, _solver_sphere):
        s = make(n)
        done = 0
        for snap in snapshots:
            s.step(snap - done)
            done = snap
            x, y, _, _ = record(s)
            xs.append(x)
            ys.append(y)
        s.close()
    x, y = torch.cat(xs), torch.cat(ys)
    g = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(x.shape[0], generator=g, device="cuda")[:max_faces]
    return x[perm].contiguous(), y[perm].contiguous()


def load_weights(path=WEIGHTS) -> np.ndarray:
    """The trained sensor shipped with the package (python -m nuc3d_b200.sensor train)."""
    return np.load(path).astype(np.float32)


def init_params(seed=0) -> np.ndarray:
    """He-uniform weights, zero biases, in the parameter order of nuc3d_gpu.h."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in ((N_IN, N_HID), (N_HID, N_HID), (N_HID, 1)):
        lim = math.sqrt(6.0 / fan_in)
        parts.append(rng.uniform(-lim, lim, fan_in * fan_out))
        parts.append(np.zeros(fan_out))
    return np.concatenate(parts).astype(np.float32)


def loss_grad(params, x, y, pos_weight=1.0, logits=None):
    """(loss, grad) on device tensors, by the library's kernels."""
    torch = _torch()
    lib = load_library()
    grad = torch.empty(N_PARAMS, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.nuc3d_sensor_loss_grad(ctypes.c_void_p(params.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                    ctypes.c_void_p(y.data_ptr()), x.shape[0], float(pos_weight),
                                    ctypes.c_void_p(grad.data_ptr()), ctypes.c_void_p(loss.data_ptr()),
                                    ctypes.c_void_p(logits.data_ptr()) if logits is not None else None,
                                    ctypes.c_void_p(st))
    if rc:
        raise RuntimeError(f"nuc3d_sensor_loss_grad failed ({rc})")
    return loss, grad


def adam_step(params, grad, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
    torch = _torch()
    lib = load_library()
    rc = lib.nuc3d_sensor_adam(*[ctypes.c_void_p(t.data_ptr()) for t in (params, grad, m, v)],
                               lr, beta1, beta2, eps, step,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if rc:
        raise RuntimeError(f"nuc3d_sensor_adam failed ({rc})")


def train(x, y, epochs=6, batch=65536, lr=3e-3, pos_weight=4.0, seed=0, log=None):
    """Adam on minibatches of `batch` faces; returns the parameters (numpy float32)."""
    torch = _torch()
    p = torch.tensor(init_params(seed), device="cuda")
    m, v = torch.zeros_like(p), torch.zeros_like(p)
    g = torch.Generator(device="cuda").manual_seed(seed + 1)
    step = 0
    n = x.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g, device="cuda")
        tot = 0.0
        for b0 in range(0, n - batch + 1, batch):
            idx = perm[b0:b0 + batch]
            loss, grad = loss_grad(p, x[idx].contiguous(), y[idx].contiguous(), pos_weight)
            step += 1
            adam_step(p, grad, m, v, step, lr=lr * (0.5 ** (ep // 2)))
            tot += float(loss.item())
        if log:
            log(f"epoch {ep}: mean loss {tot / max(1, n // batch):.5f}")
    return p.cpu().numpy()


def evaluate(params, x, y, logit_threshold=-2.0):
    """Fraction of faces sent to the linear weights and recall of the nonlinear faces
    (labels 1 predicted as needing WENO) at a logit threshold."""
    torch = _torch()
    p = torch.tensor(params, device="cuda")
    z = torch.empty(x.shape[0], dtype=torch.float32, device="cuda")
    loss_grad(p, x, y, 1.0, logits=z)
    full = z > logit_threshold
    pos = y == 1
    recall = float((full & pos).sum()) / max(1, int(pos.sum()))
    return {"linear_fraction": 1.0 - float(full.float().mean()), "recall": recall,
            "positive_fraction": float(pos.float().mean())}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train"])
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--n", type=int, default=64)
    a = ap.parse_args(argv)
    x, y = dataset(n=a.n, seed=a.seed)
    print(f"{x.shape[0]} faces, {float(y.float().mean()):.3f} need nonlinear weights", flush=True)
    params = train(x, y, seed=a.seed, log=lambda m: print(m, flush=True))
    for t in (-4.0, -3.0, -2.0, -1.0):
        print(f"threshold {t}: {evaluate(params, x, y, t)}", flush=True)
    np.save(a.out, params)
    print(f"wrote {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
