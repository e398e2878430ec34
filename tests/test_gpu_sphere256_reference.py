"""The benchmarked workload against the reference itself, at full size.

The bench's 256^3 spherical Riemann problem (FP64 Euler, WENO5-Z with the reference's
src/weno5z.cpp:80 stencil, AUSM, outlet faces, CFL 0.5) trips con2prim's energy reset
(src/physicsModel.cpp:324-332).  The reference runs it here through the project's MPI shim
as one rank per host core (a 2^k tensor-product split of the block; its multi-rank runs are
bitwise its one-rank run), for the bench's 20 + 5 steps.  The reference-order build must
reproduce the state, every step's dt and the count of reset cells bit for bit; the
throughput build must stay within 1e-10 relative max-norm of it, the north star's bar.
"""
import os

import numpy as np
import pytest

STEPS = 25


def _reference(shape, steps):
    import bench
    from oracle import refrun as R
    cores = bench.host_cores()
    nranks = 1
    while nranks * 2 <= min(cores, 64):
        nranks *= 2
    case, nr = bench.reference_case(shape, nranks)
    parts = bench.decompose(shape, nranks)
    printed = []
    out = R.run(case, "steps", steps, stdout=printed, timeout=3000)
    bs = [shape[d] // parts[d] for d in range(3)]
    q = np.empty((5, shape[2], shape[1], shape[0]))
    r = 0
    for c in range(parts[2]):
        for b in range(parts[1]):
            for a in range(parts[0]):
                q[:, c * bs[2]:(c + 1) * bs[2], b * bs[1]:(b + 1) * bs[1],
                  a * bs[0]:(a + 1) * bs[0]] = R.stack(out[r], "Q", 5)
                r += 1
    return q, out[0]["dt"], out[0]["time"], R.reset_lines(printed[0]), nr


def _ours(shape, steps, exact):
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                    gamma=1.4, cfl=0.5, exact=exact, weno5z_compat=True)
    q0, _ = C.spherical_riemann(shape)
    s = nb.Solver(cfg)
    b = s.add_block(*shape, *C.outlet_faces())
    s.set_nodes(b, *C.unit_box_nodes(shape))  # the reference's metrics, bit for bit
    s.finalize()
    s.set_q(b, q0)
    dts = []
    for _ in range(steps):
        s.step(1)
        dts.append(s.time_dt()[1])
    out = s.get_q(b), np.array(dts), s.time_dt()[0], s.energy_resets(), s.status()
    s.close()
    return out


@pytest.mark.gpu
@pytest.mark.slow
def test_sphere256_matches_reference():
    shape = (256, 256, 256)
    if not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                       "nuc3d_ref_taps")):
        pytest.skip("reference binary not built")
    qr, dtr, timer, resets_ref, nr = _reference(shape, STEPS)
    assert resets_ref > 0, "the workload is expected to trip the energy reset"
    qx, dtx, tx, resets_x, st = _ours(shape, STEPS, exact=True)
    assert st & 2, "status must report the energy reset"
    assert resets_x == resets_ref, (resets_x, resets_ref)
    assert np.array_equal(dtx, dtr) and tx == timer[-1]
    bad = int(np.sum(qx != qr))
    assert bad == 0, f"{bad} values differ; rel {np.max(np.abs(qx - qr)) / np.max(np.abs(qr)):.3g}"
    qf, dtf, _, resets_f, _ = _ours(shape, STEPS, exact=False)
    rel = float(np.max(np.abs(qf - qr)) / np.max(np.abs(qr)))
    print(f"reference {nr} ranks; resets {resets_ref}; throughput build rel max-norm {rel:.3g}, "
          f"resets {resets_f}")
    assert rel < 1e-10, rel
