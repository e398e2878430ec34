"""Run the benchmark workload at a chosen size, without timing: the target of ncu captures.

    python -m nuc3d_b200.profile_case --shape 128 --steps 1 [--exact] [--ns]
    python -m nuc3d_b200.profile_case --shape 128 --sweeps 2 [--hybrid]

Euler: spherical Riemann, WENO5-Z + AUSM, outlet faces (bench.py's workload).
--ns: Navier-Stokes Taylor-Green, WENO5-JS + LF, periodic (the small-config numerics).
--sweeps R: instead of stepping, launch each direction's right-hand-side sweep 1 + R
times (xi, then eta, then zeta: the launches bench.py times for its roofline) and
print the mean milliseconds per launch.
--hybrid: the Euler case with the learned face sensor set (hybrid WENO-Z sweeps).
"""
from __future__ import annotations

import argparse

import nuc3d_b200 as nb
from nuc3d_b200 import cases as C


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", type=int, default=128)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--exact", action="store_true")
    ap.add_argument("--ns", action="store_true")
    ap.add_argument("--sweeps", type=int, default=0)
    ap.add_argument("--hybrid", action="store_true")
    a = ap.parse_args()
    shape = (a.shape,) * 3
    if a.ns:
        cfg = nb.Config(scheme_ivs=("weno5js",) * 3, riemann="LF", model="NavierStokes3d",
                        mach=0.1, reynolds=1600.0, exact=a.exact)
        q, m = C.taylor_green(shape)
        faces = C.periodic_faces()
    else:
        cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                        exact=a.exact, weno5z_compat=True)
        q, m = C.spherical_riemann(shape)
        faces = C.outlet_faces()
    s = nb.Solver(cfg)
    b = s.add_block(*shape, *faces)
    s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, q)
    if a.hybrid:
        from nuc3d_b200 import sensor
        s.set_sensor(sensor.load_weights(), sensor.DEFAULT_THRESHOLD)
    if a.sweeps > 0:
        print([s.profile_sweep(d, a.sweeps) for d in range(3)])
        s.close()
        return
    s.step(a.steps)
    t, dt = s.time_dt()
    print(f"{shape} steps={a.steps} time={t:.6g} dt={dt:.6g} status={s.status()}")
    s.close()


if __name__ == "__main__":
    main()
