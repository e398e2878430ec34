"""The boundary-layer workload (a Mach 2.25 flat-plate boundary layer over a Gaussian
roughness bump on a tanh-stretched curvilinear mesh in 4 x 2 x 2 = 16 uneven blocks;
inlet on x-, outlet on x+, isothermal wall T_w = 1.9 on y-, outlet on y+, periodic z;
Navier-Stokes, WENO5-Z, AUSM, cd6) against the reference itself, run as 16 ranks at a
reduced size (64 x 32 x 16 cells) so that it finishes in seconds.  The wall's ghost
states (src/boundaryConditions.cpp:588-686, rho = p gamma Ma^2 / T_w, zero velocity),
the inlet's BC values (:140-274), the outlets' extrapolation (:307-459), the periodic
faces and the block-to-block halos all act on non-orthogonal metrics.  The
reference-order build must reproduce every block and every dt bit for bit after 3 steps;
the throughput build within 1e-11 relative max-norm."""
import numpy as np
import pytest

from oracle import refrun as R

SHAPE, STEPS = (64, 32, 16), 3


def _setup():
    from nuc3d_b200 import cases as C
    from nuc3d_b200.metrics import metrics_from_nodes
    blocks, types, ids, values, params = C.boundary_layer(SHAPE)
    for b in blocks:
        m = metrics_from_nodes(*b["nodes"])
        b["q"] = np.ascontiguousarray(C.prim_to_q(b["prim"], m["jac"], params["Gamma"]))
    return blocks, types, ids, values, params


def test_boundary_layer_case_layout():
    """The generator's topology: 16 blocks tiling the box, every block-to-block face
    answered by its neighbour, physical faces where the case says."""
    blocks, types, ids, values, _ = _setup()
    assert len(blocks) == 16
    assert sum(b["shape"][0] * b["shape"][1] * b["shape"][2] for b in blocks) == np.prod(SHAPE)
    assert len({b["shape"] for b in blocks}) > 1
    for r in range(16):
        for f in range(6):
            if types[r][f] >= 0:
                n = types[r][f]
                assert types[n][ids[r][f]] == r and ids[n][ids[r][f]] == f
        lo = blocks[r]["lo"]
        if lo[0] == 0:
            assert (types[r][0], ids[r][0]) == (-1, 0) and values[r][0][0] == 1.0
        if lo[1] == 0:
            assert (types[r][2], ids[r][2]) == (-1, 2)


def test_boundary_layer_full_size_partition():
    """The full 1024 x 256 x 128 case's cuts: multiples of 4 cells (the device metrics'
    requirement), summing to the grid, uneven along x."""
    from nuc3d_b200 import cases as C
    for d, (n, k) in enumerate(zip((1024, 256, 128), (4, 2, 2))):
        p = C.split_sizes(n, k, 5 + d)
        assert sum(p) == n and len(p) == k and all(v % 4 == 0 and v > 0 for v in p)
        if d == 0:
            assert len(set(p)) > 1


@pytest.fixture(scope="module")
def ref():
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    blocks, types, ids, values, params = _setup()
    topo = []
    for r in range(len(blocks)):
        lines = []
        for f in range(6):
            s = f"{types[r][f]} {ids[r][f]}"
            if types[r][f] < 0 and ids[r][f] == 0:
                s += " " + " ".join(repr(float(v)) for v in values[r][f])
            lines.append(s)
        topo.append(lines)
    case = R.Case(model="NavierStokes3d", riemann="AUSM", schemes=("weno5z",) * 3, params=params,
                  nodes=[b["nodes"] for b in blocks], bc_topo=topo, q0=[b["q"] for b in blocks],
                  start_step=1)
    out = R.run(case, "steps", STEPS, timeout=1200)
    return [R.stack(d, "Q", 5) for d in out], out[0]["dt"], out[0]["time"], out[0]["res"]


def _gpu(exact):
    import nuc3d_b200 as nb
    blocks, types, ids, values, params = _setup()
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="NavierStokes3d",
                            reynolds=params["Reynolds"], mach=params["Mach"],
                            t_wall=params["T_wall"], exact=exact))
    for r, b in enumerate(blocks):
        s.add_block(*b["shape"], types[r], ids[r], values[r])
    for r, b in enumerate(blocks):
        s.set_nodes(r, *b["nodes"])
    s.finalize()
    for r, b in enumerate(blocks):
        s.set_q(r, b["q"])
    dts = []
    for _ in range(STEPS):
        s.step(1)
        dts.append(s.time_dt()[1])
    out = [s.get_q(r) for r in range(len(blocks))], np.array(dts), s.time_dt()[0], s.residual()
    s.close()
    return out


@pytest.mark.gpu
def test_boundary_layer_bitwise(ref):
    q, dts, t, res = _gpu(exact=True)
    qr, dtr, tr, resr = ref
    assert np.array_equal(dts, dtr) and t == tr[-1]
    for r in range(len(q)):
        assert np.array_equal(q[r], qr[r]), (r, float(np.max(np.abs(q[r] - qr[r]))))
    assert res == resr[-1]


@pytest.mark.gpu
def test_boundary_layer_fast(ref):
    q, _, _, _ = _gpu(exact=False)
    qr = ref[0]
    scale = max(float(np.max(np.abs(a))) for a in qr)
    err = max(float(np.max(np.abs(a - b))) for a, b in zip(q, qr))
    assert err <= 1e-11 * scale, err / scale
