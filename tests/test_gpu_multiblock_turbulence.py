"""Many uneven blocks: decaying isotropic turbulence in a periodic 2 pi box cut into
2 x 3 x 4 = 24 blocks whose sizes along each axis are drawn with a fixed seed (the
structure of the reference's batched multi-block configuration, block sizes scaled down
so that the reference finishes in seconds), Navier-Stokes, WENO5-Z + AUSM, cd6.

The reference runs as 24 MPI ranks (one block each, the project's shared-memory MPI
shim); the GPU advances the 24 blocks in one context, halos read from the neighbour
blocks.  The reference-order build must reproduce every block bit for bit after 3
TVD-RK3 steps, with the same dt; the throughput build within 1e-11 relative.
"""
import math

import numpy as np
import pytest

from oracle import refrun as R

PARTS_SEED, FIELD_SEED, STEPS, MT = 1, 2, 3, 0.6


def _setup():
    from nuc3d_b200 import cases as C
    from nuc3d_b200.metrics import metrics_from_nodes
    parts = C.uneven_blocks(sizes=(8, 12, 16, 20), seed=PARTS_SEED)
    n = [sum(p) for p in parts]
    x, y, z = R.box_nodes(*n, hi=(2.0 * math.pi,) * 3)
    prim, reynolds = C.isotropic_turbulence(tuple(n), seed=FIELD_SEED, mt=MT)
    types, ids = C.block_topology(parts)
    off = [np.concatenate([[0], np.cumsum(p)]) for p in parts]
    blocks = []
    for c in range(len(parts[2])):
        for b in range(len(parts[1])):
            for a in range(len(parts[0])):
                lo = (off[0][a], off[1][b], off[2][c])
                hi = (off[0][a + 1], off[1][b + 1], off[2][c + 1])
                nsl = tuple(slice(lo[d], hi[d] + 1) for d in (2, 1, 0))
                csl = tuple(slice(lo[d], hi[d]) for d in (2, 1, 0))
                xyz = tuple(arr[nsl] for arr in (x, y, z))
                m = metrics_from_nodes(*xyz)
                q = C.prim_to_q(prim[(slice(None),) + csl], m["jac"], 1.4)
                blocks.append(dict(shape=tuple(int(hi[d] - lo[d]) for d in range(3)),
                                   nodes=xyz, q=np.ascontiguousarray(q)))
    params = {"Reynolds": reynolds, "Mach": MT, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
              "T_inf": 288.0, "T_wall": 1.0}
    return blocks, types, ids, params


@pytest.fixture(scope="module")
def case():
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    blocks, types, ids, params = _setup()
    topo = [[f"{types[r][f]} {ids[r][f]}" for f in range(6)] for r in range(len(blocks))]
    ref = R.Case(model="NavierStokes3d", riemann="AUSM", schemes=("weno5z",) * 3, params=params,
                 nodes=[b["nodes"] for b in blocks], bc_topo=topo, q0=[b["q"] for b in blocks],
                 start_step=1)
    out = R.run(ref, "steps", STEPS, timeout=1200)
    return blocks, types, ids, params, [R.stack(d, "Q", 5) for d in out], out[0]["dt"], out[0]["time"]


def _gpu(blocks, types, ids, params, exact):
    import nuc3d_b200 as nb
    cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                    reynolds=params["Reynolds"], mach=MT, prandtl=0.72, exact=exact)
    s = nb.Solver(cfg)
    for r, b in enumerate(blocks):
        s.add_block(*b["shape"], types[r], ids[r])
    for r, b in enumerate(blocks):
        s.set_mesh(r, *b["nodes"])
    s.finalize()
    for r, b in enumerate(blocks):
        s.set_q(r, b["q"])
    s.step(STEPS)
    return [s.get_q(r) for r in range(len(blocks))], s.time_dt()


@pytest.mark.gpu
def test_uneven_blocks_bitwise(case):
    blocks, types, ids, params, qref, dts, times = case
    q, (t, dt) = _gpu(blocks, types, ids, params, exact=True)
    assert t == times[-1] and dt == dts[-1]
    for r in range(len(blocks)):
        assert np.array_equal(q[r], qref[r]), (r, float(np.max(np.abs(q[r] - qref[r]))))


@pytest.mark.gpu
def test_uneven_blocks_fast(case):
    blocks, types, ids, params, qref, dts, times = case
    q, _ = _gpu(blocks, types, ids, params, exact=False)
    scale = max(float(np.max(np.abs(a))) for a in qref)
    err = max(float(np.max(np.abs(a - b))) for a, b in zip(q, qref))
    assert err <= 1e-11 * scale, err / scale


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [True, False])
def test_solve_host_by_block_equals_device_steps(exact):
    """nuc3d_solve_host on the 24 uneven blocks (one host array each): stage 2 runs block by
    block after every block's ghost fluxes and gradients, and each block's download starts
    after its own zeta sweep.  The same 3 steps as on the device-resident state, bit for bit:
    every block, time, dt and the residual; the whole-step path (pipeline off) too."""
    import nuc3d_b200 as nb
    blocks, types, ids, params = _setup()

    def make():
        cfg = nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                        reynolds=params["Reynolds"], mach=MT, prandtl=0.72, exact=exact)
        s = nb.Solver(cfg)
        for r, b in enumerate(blocks):
            s.add_block(*b["shape"], types[r], ids[r])
        for r, b in enumerate(blocks):
            s.set_mesh(r, *b["nodes"])
        s.finalize()
        for r, b in enumerate(blocks):
            s.set_q(r, b["q"])
        return s

    s1 = make()
    s1.step(STEPS)
    ref = [s1.get_q(r) for r in range(len(blocks))], s1.time_dt(), s1.residual()
    s1.close()
    for pipe in (True, False):
        s2 = make()
        s2.set_host_pipeline(pipe)
        host = [np.ascontiguousarray(b["q"]).copy() for b in blocks]
        s2.solve_host([h.ctypes.data for h in host], STEPS)
        for r in range(len(blocks)):
            assert np.array_equal(host[r], ref[0][r]), (pipe, r)
        assert s2.time_dt() == ref[1] and s2.residual() == ref[2]
        s2.close()
