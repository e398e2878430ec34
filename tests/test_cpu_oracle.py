"""The C restatement (oracle/nuc3d_oracle.c) reproduces the reference's golden vectors
bit for bit: metrics, one right-hand side, dt, the state after 1 and n steps, and the
postproc::solveQ diagnostics (totals and fields) of that state."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G


def oracle_run(g):
    r = O.Run(g.cfg["schemes"], g.cfg["riemann"], g.cfg["model"], g.cfg["params"],
              vis=G.vis(g))
    t, i, v = G.bc_arrays(g)
    r.add_block(O.metrics(*G.nodes(g)), t, i, v, g.q0)
    return r


def test_oracle_metrics_bitwise():
    g = G.load("tgv_ns_weno5js_lf")
    m = O.metrics(*G.nodes(g))
    assert np.array_equal(m["jac"], g.metrics_jac)
    for nm in ("xi_xyz", "eta_xyz", "zeta_xyz", "dxyz"):
        assert np.array_equal(m[nm], g.data[f"metrics_{nm}"]), nm


@pytest.mark.parametrize("name", G.names())
def test_oracle_rhs_bitwise(name):
    g = G.load(name)
    dt, rhs = oracle_run(g).rhs()
    assert dt == g.dt_local[0]
    assert np.array_equal(rhs[0], g.rhs), np.max(np.abs(rhs[0] - g.rhs))


@pytest.mark.parametrize("name", G.names())
def test_oracle_steps_bitwise(name):
    g = G.load(name)
    r = oracle_run(g)
    dt, t = r.step(1)
    assert np.array_equal(r.q(0), g.q1)
    assert dt[0] == g.dt[0]
    n = int(g.cfg["nsteps"])
    r = oracle_run(g)
    dt, t = r.step(n)
    assert np.array_equal(r.q(0), g.qn), np.max(np.abs(r.q(0) - g.qn))
    assert np.array_equal(dt, g.dt) and t == g.time[-1]
    assert np.array_equal(r.res, g.res), (r.res, g.res)  # block::RES after each step


@pytest.mark.parametrize("name", G.diag_names())
def test_oracle_diag_bitwise(name):
    g, d = G.load(name), G.load_diag(name)
    r = O.Run(g.cfg["schemes"], g.cfg["riemann"], g.cfg["model"], g.cfg["params"], vis=G.vis(g))
    t, i, v = G.bc_arrays(g)
    r.add_block(O.metrics(*G.nodes(g)), t, i, v, g.qn)
    ens, kin, f = r.diag()
    assert ens == d["enstrophy"][0] and kin == d["kinetic"][0], (ens - d["enstrophy"][0], kin - d["kinetic"][0])
    assert np.array_equal(f[0], d["fields"]), np.max(np.abs(f[0] - d["fields"]))


def test_oracle_diag_two_blocks_bitwise():
    """The reference run as two ranks: fields equal the single block's, totals are the
    block sums added in rank order."""
    g, d = G.load("tgv_ns_weno5js_lf"), G.load_diag("tgv_ns_weno5js_lf.2ranks")
    m = O.metrics(*G.nodes(g))
    h = g.cfg["shape"][0] // 2
    keys = ("jac", "xi_xyz", "eta_xyz", "zeta_xyz", "dxyz")
    left, right = G.split_xi([m[k] for k in keys] + [g.qn], h)
    r = O.Run(g.cfg["schemes"], g.cfg["riemann"], g.cfg["model"], g.cfg["params"])
    for b, part in enumerate((left, right)):
        mb = {k: np.ascontiguousarray(a) for k, a in zip(keys, part[:5])}
        r.add_block(mb, G.TWO_BLOCK_TYPES[b], G.TWO_BLOCK_IDS[b], None, np.ascontiguousarray(part[5]))
    ens, kin, f = r.diag()
    assert ens == d["enstrophy"][0] and kin == d["kinetic"][0]
    assert np.array_equal(np.concatenate(f, axis=-1), d["fields"])


@pytest.mark.parametrize("name", G.multi_names())
def test_oracle_two_ranks_bitwise(name):
    """The reference run as two ranks cut along xi, n steps: each block's own system
    (hccs77 solves per block, so this is not the one-rank result)."""
    g, mr = G.load(name), G.load_multi(name)
    m = O.metrics(*G.nodes(g))
    h = g.cfg["shape"][0] // 2
    keys = ("jac", "xi_xyz", "eta_xyz", "zeta_xyz", "dxyz")
    left, right = G.split_xi([m[k] for k in keys] + [mr["q0"]], h)
    r = O.Run(g.cfg["schemes"], g.cfg["riemann"], g.cfg["model"], g.cfg["params"], vis=G.vis(g))
    for b, part in enumerate((left, right)):
        mb = {k: np.ascontiguousarray(a) for k, a in zip(keys, part[:5])}
        t, i, v = G.two_block_bc(g, b)
        r.add_block(mb, t, i, v, np.ascontiguousarray(part[5]))
    dt, t = r.step(int(mr["nsteps"][0]))
    assert np.array_equal(dt, mr["dt"]) and t == mr["time"][-1]
    q = np.concatenate([r.q(0), r.q(1)], axis=-1)
    assert np.array_equal(q, mr["qn"]), np.max(np.abs(q - mr["qn"]))
    assert np.array_equal(r.res, mr["res"])  # MPI_Allreduce MAX of the ranks' residuals
    assert not np.array_equal(q, g.qn)


def test_oracle_uneven_blocks_bitwise():
    """24 uneven blocks of decaying turbulence (tests/test_gpu_multiblock_turbulence.py):
    the restatement against the reference run as 24 ranks, 3 steps."""
    from oracle import refrun as R
    from tests import test_gpu_multiblock_turbulence as T
    if not (R.REF_BIN_DIR / "nuc3d_ref_taps").exists():
        pytest.skip("reference binaries not built (make -C oracle ref)")
    blocks, types, ids, params = T._setup()
    topo = [[f"{types[r][f]} {ids[r][f]}" for f in range(6)] for r in range(len(blocks))]
    ref = R.Case(model="NavierStokes3d", riemann="AUSM", schemes=("weno5z",) * 3, params=params,
                 nodes=[b["nodes"] for b in blocks], bc_topo=topo, q0=[b["q"] for b in blocks],
                 start_step=1)
    out = R.run(ref, "steps", T.STEPS, timeout=1200)
    r = O.Run(("weno5z",) * 3, "AUSM", "NavierStokes3d", params)
    for i, b in enumerate(blocks):
        r.add_block(O.metrics(*b["nodes"]), types[i], ids[i], None, b["q"])
    dt, t = r.step(T.STEPS)
    assert np.array_equal(dt, out[0]["dt"])
    for i in range(len(blocks)):
        assert np.array_equal(r.q(i), R.stack(out[i], "Q", 5)), i
