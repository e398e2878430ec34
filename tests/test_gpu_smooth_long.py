"""A long run of a smooth, stable flow against the reference itself: a weak isentropic
pressure pulse (amplitude 0.05) in a periodic unit box of 48^3 cells, FP64 Euler,
WENO5-JS, AUSM, TVD-RK3 at CFL 0.5, 100 steps (to t = 1.04: the acoustic waves cross the
box once).  The reference runs as 8 ranks (2 x 2 x 2 blocks of 24^3
through the project's MPI shim); the GPU advances the same 8 blocks in one context.  The
reference-order build must reproduce every block and every dt bit for bit; the throughput
build (FMA contraction, one division per face) must stay within 1e-10 relative max-norm
after all 100 steps: on a smooth flow its round-off does not grow into the solution."""
import numpy as np
import pytest

from oracle import refrun as R

N, STEPS, AMP = 48, 100, 0.05


def _setup():
    from nuc3d_b200 import cases as C
    shape = (N, N, N)
    parts = [[N // 2, N // 2]] * 3
    x, y, z = C.unit_box_nodes(shape)
    prim_q, _ = C.gaussian_pulse(shape, amp=AMP)  # U/J of the whole box
    types, ids = C.block_topology(parts)
    h = N // 2
    blocks = []
    for c in range(2):
        for b in range(2):
            for a in range(2):
                nsl = (slice(c * h, c * h + h + 1), slice(b * h, b * h + h + 1), slice(a * h, a * h + h + 1))
                csl = (slice(None), slice(c * h, c * h + h), slice(b * h, b * h + h), slice(a * h, a * h + h))
                xyz = tuple(arr[nsl] for arr in (x, y, z))
                blocks.append(dict(nodes=xyz, q=np.ascontiguousarray(prim_q[csl])))
    return blocks, types, ids


@pytest.fixture(scope="module")
def ref():
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    blocks, types, ids = _setup()
    topo = [[f"{types[r][f]} {ids[r][f]}" for f in range(6)] for r in range(len(blocks))]
    case = R.Case(model="Euler3d", riemann="AUSM", schemes=("weno5js",) * 3,
                  params={"Reynolds": 1000.0, "Mach": 1.0, "Pt": 0.72, "Gamma": 1.4,
                          "T_ref": 110.4, "T_inf": 288.0, "T_wall": 1.0},
                  nodes=[b["nodes"] for b in blocks], bc_topo=topo, q0=[b["q"] for b in blocks],
                  start_step=1)
    out = R.run(case, "steps", STEPS, timeout=1800)
    return [R.stack(d, "Q", 5) for d in out], out[0]["dt"], out[0]["time"]


def _gpu(exact):
    import nuc3d_b200 as nb
    blocks, types, ids = _setup()
    s = nb.Solver(nb.Config(scheme_ivs=("weno5js",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                            exact=exact))
    for r in range(len(blocks)):
        s.add_block(N // 2, N // 2, N // 2, types[r], ids[r])
    for r, b in enumerate(blocks):
        s.set_nodes(r, *b["nodes"])
    s.finalize()
    for r, b in enumerate(blocks):
        s.set_q(r, b["q"])
    dts = []
    for _ in range(STEPS):
        s.step(1)
        dts.append(s.time_dt()[1])
    out = [s.get_q(r) for r in range(len(blocks))], np.array(dts), s.time_dt()[0]
    s.close()
    return out


@pytest.mark.gpu
def test_smooth_long_bitwise(ref):
    q, dts, t = _gpu(exact=True)
    qr, dtr, tr = ref
    assert np.array_equal(dts, dtr) and t == tr[-1]
    for r in range(len(q)):
        assert np.array_equal(q[r], qr[r]), (r, float(np.max(np.abs(q[r] - qr[r]))))


@pytest.mark.gpu
def test_smooth_long_fast_within_1e10(ref):
    q, dts, _ = _gpu(exact=False)
    qr, dtr, _ = ref
    scale = max(float(np.max(np.abs(a))) for a in qr)
    err = max(float(np.max(np.abs(a - b))) for a, b in zip(q, qr))
    assert err <= 1e-10 * scale, err / scale
    assert np.max(np.abs(dts - dtr) / dtr) <= 1e-12
