"""Hybrid WENO-Z: the sweep's tensor-core sensor inference and its per-face choice of
weights, on a periodic Lax-Friedrichs Euler block (every face interior).

  threshold -inf  no face takes the linear weights: the plain throughput RHS
  threshold +inf  every face does: the numpy RHS with linear weights
  threshold t     the faces whose logit, by the training forward, lies below t: the numpy
                  RHS with exactly those faces linear (t sits in a gap of the logits, so
                  BF16 rounding differences between the two paths cannot flip a face)
"""
import numpy as np
import pytest

from tests import golden_cases as G
from tests import sensor_np as SN

GAMMA = 1.4


def _solver(sensor=None, thr=0.0):
    import nuc3d_b200 as nb
    g = G.load("tgv_ns_weno5js_lf")
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="LF", model="Euler3d", mach=0.1,
                            exact=False, weno5z_compat=True))
    nx, ny, nz = g.cfg["shape"]
    b = s.add_block(nx, ny, nz, *G.bc_arrays(g)[:2])
    m = s.set_mesh(b, *G.nodes(g))
    s.finalize()
    s.set_q(b, g.qn)
    if sensor is not None:
        s.set_sensor(sensor, thr)
    return s, m, g.qn


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.gpu
def test_hybrid_never_linear_is_plain():
    from nuc3d_b200 import sensor as S
    s0, _, _ = _solver()
    s0.rhs()
    plain = s0.get_rhs(0)
    s1, _, _ = _solver(S.load_weights(), -np.inf)
    s1.rhs()
    assert _rel(s1.get_rhs(0), plain) <= 1e-15


@pytest.mark.gpu
def test_hybrid_always_linear_matches_numpy():
    from nuc3d_b200 import sensor as S
    s, m, q = _solver(S.load_weights(), np.inf)
    s.rhs()
    ref = SN.hybrid_rhs(q, m, GAMMA, True, [np.ones(q.shape[1:], bool)] * 3)
    assert _rel(s.get_rhs(0), ref) <= 1e-12


@pytest.mark.gpu
def test_hybrid_decisions_follow_the_trained_network():
    import torch
    from nuc3d_b200 import sensor as S
    params = S.load_weights()
    s, m, q = _solver()
    feats = [SN.features(q, m, d, GAMMA, True)[0] for d in range(3)]
    x = torch.tensor(np.concatenate([f.reshape(-1, 19) for f in feats]).astype(np.float32), device="cuda")
    z = torch.empty(x.shape[0], dtype=torch.float32, device="cuda")
    S.loss_grad(torch.tensor(params, device="cuda"), x, torch.zeros(x.shape[0], dtype=torch.uint8,
                                                                    device="cuda"), 1.0, logits=z)
    zs = np.sort(z.cpu().numpy())
    gaps = np.diff(zs)
    k = int(np.argmax(np.where((np.arange(len(gaps)) > len(zs) // 10) &
                               (np.arange(len(gaps)) < 9 * len(zs) // 10), gaps, 0)))
    thr = float(0.5 * (zs[k] + zs[k + 1]))
    assert gaps[k] > 0.02, gaps[k]
    zz = z.cpu().numpy()
    n = [f.shape[0] * f.shape[1] * f.shape[2] for f in feats]
    masks = [zz[sum(n[:d]):sum(n[:d + 1])].reshape(feats[d].shape[:3]) < thr for d in range(3)]
    frac = float(np.mean(np.concatenate([mk.ravel() for mk in masks])))
    assert 0.05 < frac < 0.95, frac     # both kinds of faces present
    sh, _, _ = _solver(params, thr)
    sh.rhs()
    ref = SN.hybrid_rhs(q, m, GAMMA, True, masks)
    assert _rel(sh.get_rhs(0), ref) <= 1e-12


@pytest.mark.gpu
def test_theta_switch_decisions():
    """hccs's theta switch as the decision (nuc3d_set_sensor_theta): theta_min above 1
    never selects the linear weights (plain), 0 always does, and a theta_min inside a gap
    of the faces' thetas selects exactly the faces whose numpy theta reaches it."""
    s0, _, _ = _solver()
    s0.rhs()
    plain = s0.get_rhs(0)
    s, m, q = _solver()
    s.set_sensor_theta(2.0)
    s.rhs()
    assert _rel(s.get_rhs(0), plain) <= 1e-15
    s.set_sensor_theta(0.0)
    s.rhs()
    assert _rel(s.get_rhs(0), SN.hybrid_rhs(q, m, GAMMA, True, [np.ones(q.shape[1:], bool)] * 3)) <= 1e-12
    th = [SN.theta_faces(q, m, d, GAMMA) for d in range(3)]
    ts = np.sort(np.concatenate([t.ravel() for t in th]))
    gaps = np.diff(ts)
    idx = np.arange(len(gaps))
    k = int(np.argmax(np.where((idx > len(ts) // 10) & (idx < 9 * len(ts) // 10), gaps, 0)))
    tmin = float(0.5 * (ts[k] + ts[k + 1]))
    assert gaps[k] > 1e-6 * max(tmin, 1e-300), gaps[k]
    masks = [t >= tmin for t in th]
    frac = float(np.mean(np.concatenate([mk.ravel() for mk in masks])))
    assert 0.05 < frac < 0.95, frac
    s.set_sensor_theta(tmin)
    s.rhs()
    assert _rel(s.get_rhs(0), SN.hybrid_rhs(q, m, GAMMA, True, masks)) <= 1e-12
    s.set_sensor(None)
    s.rhs()
    assert _rel(s.get_rhs(0), plain) <= 1e-15


@pytest.mark.gpu
def test_exact_build_refuses_the_sensor():
    import nuc3d_b200 as nb
    from nuc3d_b200 import sensor as S
    g = G.load("tgv_ns_weno5js_lf")
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="LF", model="Euler3d", exact=True))
    nx, ny, nz = g.cfg["shape"]
    b = s.add_block(nx, ny, nz, *G.bc_arrays(g)[:2])
    s.set_mesh(b, *G.nodes(g))
    s.finalize()
    with pytest.raises(nb.Nuc3dError) as e:
        s.set_sensor(S.load_weights(), 0.0)
    assert e.value.code == 5
    with pytest.raises(nb.Nuc3dError) as e:
        s.set_sensor_theta(0.5)
    assert e.value.code == 5


def _sphere_run(n, steps, sensor=None, thr=-2.0):
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    q, m = C.spherical_riemann((n, n, n))
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                            exact=False))
    b = s.add_block(n, n, n, *C.outlet_faces())
    s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
    s.finalize()
    s.set_q(b, q)
    if sensor is not None:
        s.set_sensor(sensor, thr)
    try:
        s.step(steps)
        return s.get_q(b)[0] * m["jac"]   # density
    except nb.Nuc3dError:
        return None                       # the run failed (negative pressure / non-finite)


@pytest.mark.gpu
@pytest.mark.slow
def test_hybrid_shock_error_and_what_the_network_buys():
    """Spherical Riemann problem, 64^3, 60 steps (the shock crosses several cells).  With
    the trained sensor at the default threshold the L1 density error against plain WENO-Z
    stays below 1e-3; all faces on linear weights (the method without the network) are
    off by about 20% here and fail outright (non-finite state) at 128^3."""
    from nuc3d_b200 import sensor as S
    plain = _sphere_run(64, 60)
    hyb = _sphere_run(64, 60, S.load_weights(), S.DEFAULT_THRESHOLD)
    lin = _sphere_run(64, 60, S.load_weights(), np.inf)
    l1 = lambda a: float(np.abs(a - plain).sum() / np.abs(plain).sum())  # noqa: E731
    assert hyb is not None and l1(hyb) <= 1e-3, l1(hyb)
    assert lin is None or l1(lin) >= 10.0 * max(l1(hyb), 1e-6), (l1(lin), l1(hyb))
