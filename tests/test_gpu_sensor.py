"""The learned face sensor's CUDA kernels: features and labels against a numpy
restatement, loss and gradients against torch fp32 autograd, the Adam step against its
formula.
"""
import math

import numpy as np
import pytest

from tests import golden_cases as G


def _torch_reference(params, x, y, pos_weight):
    """The network of nuc3d_gpu.h in torch fp32 on the CPU, with the kernels' BF16
    roundings (gradients pass them straight through)."""
    import torch
    P = params.detach().cpu().clone().requires_grad_(True)
    W1, b1 = P[:608].view(32, 19), P[608:640]
    W2, b2 = P[640:1664].view(32, 32), P[1664:1696]
    W3, b3 = P[1696:1728], P[1728]
    bfr = lambda t: t.to(torch.bfloat16).to(torch.float32)  # noqa: E731
    xr = bfr(x.cpu())
    h1 = bfr(torch.relu(xr @ bfr(W1).T + bfr(b1)))
    h2 = bfr(torch.relu(h1 @ bfr(W2).T + bfr(b2)))
    z = h2 @ bfr(W3) + bfr(b3)
    t = y.cpu().float()
    sp = torch.nn.functional.softplus
    loss = (pos_weight * t * sp(-z) + (1.0 - t) * sp(z)).mean()
    loss.backward()
    return float(loss.detach()), P.grad, z.detach()


@pytest.mark.gpu
def test_loss_and_gradient_match_torch():
    import torch
    from nuc3d_b200 import sensor as S
    rng = np.random.default_rng(5)
    n = 3001  # not a multiple of the 64-sample tile
    p = S.init_params(3)
    p[608:640] = rng.normal(0, 0.1, 32)          # non-zero biases too
    p[1664:1696] = rng.normal(0, 0.1, 32)
    p[1728] = 0.3
    params = torch.tensor(p, device="cuda")
    x = torch.tensor(rng.uniform(0, 1, (n, 19)).astype(np.float32), device="cuda")
    y = torch.tensor((rng.uniform(0, 1, n) < 0.3).astype(np.uint8), device="cuda")
    z = torch.empty(n, dtype=torch.float32, device="cuda")
    loss, grad = S.loss_grad(params, x, y, pos_weight=3.0, logits=z)
    torch.cuda.synchronize()
    lref, gref, zref = _torch_reference(params, x, y, 3.0)
    # FP32 sums in another order can flip a BF16 rounding of a hidden activation (a step of
    # 2^-8 relative), so logits and gradients agree to that level, not to FP32 round-off
    assert abs(float(loss) - lref) <= 1e-3 * abs(lref)
    assert float((z.cpu() - zref).abs().max()) <= 1e-2 * (1.0 + float(zref.abs().max()))
    g = grad.cpu()
    scale = float(gref.abs().max())
    assert float((g - gref).abs().max()) <= 2e-2 * scale, float((g - gref).abs().max()) / scale
    # and without any flip the gradient direction is the same
    cos = float((g * gref).sum() / (g.norm() * gref.norm()))
    assert cos > 0.9999, cos


@pytest.mark.gpu
def test_adam_step_matches_formula():
    import torch
    from nuc3d_b200 import sensor as S
    rng = np.random.default_rng(1)
    p0 = rng.normal(0, 1, 1729).astype(np.float32)
    g = rng.normal(0, 1, 1729).astype(np.float32)
    m0 = rng.normal(0, 0.1, 1729).astype(np.float32)
    v0 = rng.uniform(0, 0.1, 1729).astype(np.float32)
    tp, tg, tm, tv = (torch.tensor(a, device="cuda") for a in (p0, g, m0, v0))
    S.adam_step(tp, tg, tm, tv, step=3, lr=1e-2)
    torch.cuda.synchronize()
    m = 0.9 * m0 + 0.1 * g
    v = 0.999 * v0 + 0.001 * g * g
    p = p0 - 1e-2 * (m / (1 - 0.9 ** 3)) / (np.sqrt(v / (1 - 0.999 ** 3)) + 1e-8)
    assert np.allclose(tp.cpu().numpy(), p, rtol=1e-5, atol=1e-6)


def _numpy_features(q, m, d, gamma, compat):
    """Features and deviations on the face grid (face L of the periodic line = face 0)."""
    from tests import sensor_np as SN
    X, dev = SN.features(q, m, d, gamma, compat)
    ax = 2 - d
    X = np.concatenate([X, np.take(X, [0], axis=ax)], axis=ax)
    dev = np.concatenate([dev, np.take(dev, [0], axis=ax)], axis=ax)
    return X.reshape(-1, 19), dev.reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("d", [0, 1, 2])
def test_record_matches_numpy(d):
    import torch
    import nuc3d_b200 as nb
    from nuc3d_b200 import sensor as S
    g = G.load("tgv_ns_weno5js_lf")
    s = nb.Solver(nb.Config(scheme_ivs=("weno5z",) * 3, riemann="LF", model="Euler3d", mach=0.1,
                            exact=True, weno5z_compat=True))
    nx, ny, nz = g.cfg["shape"]
    b = s.add_block(nx, ny, nz, *G.bc_arrays(g)[:2])
    m = s.set_mesh(b, *G.nodes(g))
    s.finalize()
    s.set_q(b, g.qn)
    x, y, where, counts = S.record(s, dirs=(d,), cap=1 << 16)
    X, dev = _numpy_features(g.qn, m, d, 1.4, True)
    wh = where.cpu().numpy()
    assert counts[0] == X.shape[0] and len(np.unique(wh)) == counts[0]  # every face once
    assert np.max(np.abs(x.cpu().numpy() - X[wh])) <= 1e-5
    lab = y.cpu().numpy().astype(bool)
    clear = np.abs(dev[wh] - 0.05) > 1e-9
    assert np.array_equal(lab[clear], dev[wh][clear] > 0.05)
