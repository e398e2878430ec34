"""numpy restatement for the face-sensor tests: Lax-Friedrichs split fluxes of a periodic
block (src/physicsModel.cpp:940-979), the sensor features and labels, and WENO5 face
values with WENO-Z or linear weights (src/weno5z.cpp:74-109)."""
import numpy as np

C5 = (0.1, 0.6, 0.3)


def lf_split(q, m, d, gamma):
    jac = m["jac"]
    rho = q[0] * jac
    u, v, w = q[1] / rho * jac, q[2] / rho * jac, q[3] / rho * jac
    E = q[4] * jac
    p = (E - 0.5 * rho * (u * u + v * v + w * w)) * (gamma - 1.0)
    c = np.sqrt(np.abs(gamma * p / rho))
    xx, xy, xz = m[("xi_xyz", "eta_xyz", "zeta_xyz")[d]]
    U0 = xx * u + xy * v + xz * w
    M = np.abs(U0) + c * np.sqrt(xx * xx + xy * xy + xz * xz)
    F = [U0 * q[0], U0 * q[1] + xx * p / jac, U0 * q[2] + xy * p / jac, U0 * q[3] + xz * p / jac,
         U0 * (q[4] + p / jac)]
    return ([0.5 * (F[k] + M * q[k]) for k in range(5)], [0.5 * (F[k] - M * q[k]) for k in range(5)],
            rho, p)


def parts(f0, f1, f2, f3, f4, comp):
    is0 = 13 / 12 * (f0 - 2 * f1 + f2) ** 2 + 0.25 * (f0 - 4 * f1 + 3 * f2) ** 2
    is1 = 13 / 12 * (f1 - 2 * f2 + f3) ** 2 + 0.25 * (f1 - f3) ** 2
    is2 = 13 / 12 * (f2 - 2 * f3 + np.where(comp, f3, f4)) ** 2 + 0.25 * (3 * f2 - 4 * f3 + f4) ** 2
    q0 = 1 / 3 * f0 - 7 / 6 * f1 + 11 / 6 * f2
    q1 = -1 / 6 * f1 + 5 / 6 * f2 + 1 / 3 * f3
    q2 = 1 / 3 * f2 + 5 / 6 * f3 - 1 / 6 * f4
    return (is0, is1, is2), (q0, q1, q2)


def weno5z_weights(f, comp):
    (is0, is1, is2), qs = parts(*f, comp)
    tau = np.abs(is2 - is0)
    a = [C5[k] * (1 + (tau / (s + 1e-6)) ** 2) for k, s in enumerate((is0, is1, is2))]
    tot = a[0] + a[1] + a[2]
    return [ak / tot for ak in a], qs


def weno5z_value(f, comp):
    om, qs = weno5z_weights(f, comp)
    return om[0] * qs[0] + om[1] * qs[1] + om[2] * qs[2]


def linear_value(f):
    _, qs = parts(*f, False)
    return C5[0] * qs[0] + C5[1] * qs[1] + C5[2] * qs[2]


class PeriodicLine:
    """Values at line offsets from each face of direction d (face f = cells f-1 | f);
    arrays on the (periodic) cell grid, faces 0 .. L-1."""

    def __init__(self, d, shape):
        self.ax = 2 - d
        self.L = shape[self.ax]

    def at(self, a, c):
        return np.roll(a, -c, axis=self.ax)

    def compat(self, compat):
        idx = np.arange(self.L).reshape([-1 if i == self.ax else 1 for i in range(3)])
        return compat & (idx >= 3) & (idx <= self.L - 3)


def features(q, m, d, gamma, compat):
    """Features (faces 0..L-1 of the periodic line, shape (..., 19)) and label deviations."""
    Fp, Fn, rho, p = lf_split(q, m, d, gamma)
    ln = PeriodicLine(d, rho.shape)
    cz = ln.compat(compat)
    feat, dev = [], np.zeros_like(rho)
    for v in range(5):
        f = [ln.at(Fp[v], c) for c in (-3, -2, -1, 0, 1)]
        (b0, b1, b2), _ = parts(*f, False)
        den = b0 + b1 + b2 + 1e-6
        feat += [b0 / den, b1 / den, b2 / den]
        om, _ = weno5z_weights(f, cz)
        dev = np.maximum(dev, np.maximum.reduce([np.abs(om[k] - C5[k]) for k in range(3)]))
        n_ = [ln.at(Fn[v], c) for c in (2, 1, 0, -1, -2)]
        om, _ = weno5z_weights(n_, np.zeros_like(cz))
        dev = np.maximum(dev, np.maximum.reduce([np.abs(om[k] - C5[k]) for k in range(3)]))
    rj = lambda a, b: np.abs(b - a) / (np.abs(a) + np.abs(b) + 1e-300)  # noqa: E731
    feat += [rj(ln.at(rho, -1), ln.at(rho, 0)), rj(ln.at(p, -1), ln.at(p, 0))]
    feat += [np.maximum.reduce([rj(ln.at(rho, c), ln.at(rho, c + 1)) for c in range(-3, 2)]),
             np.maximum.reduce([rj(ln.at(p, c), ln.at(p, c + 1)) for c in range(-3, 2)])]
    return np.stack(feat, axis=-1), dev


def hybrid_rhs(q, m, gamma, compat, linear_mask):
    """RHS of a periodic LF Euler block with WENO-Z, linear weights where linear_mask[d]
    (faces 0..L-1 of direction d) is true."""
    rhs = np.zeros_like(q)
    for d in range(3):
        Fp, Fn, rho, _ = lf_split(q, m, d, gamma)
        ln = PeriodicLine(d, rho.shape)
        cz = ln.compat(compat)
        for v in range(5):
            fp = [ln.at(Fp[v], c) for c in (-3, -2, -1, 0, 1)]
            fn = [ln.at(Fn[v], c) for c in (2, 1, 0, -1, -2)]
            full = weno5z_value(fp, cz) + weno5z_value(fn, np.zeros_like(cz))
            lin = linear_value(fp) + linear_value(fn)
            h = np.where(linear_mask[d], lin, full)
            rhs[v] += ln.at(h, 1) - h
    return rhs


def theta_stencil(f0, f1, f2, f3, f4):
    """hccs's switch theta = 1 / (1 + (sum alpha - 1)^2), CRWENO5-Z numerators with eps
    1e-40 (src/hccs.cpp:154-181)."""
    (is0, is1, is2), _ = parts(f0, f1, f2, f3, f4, False)
    tau = np.abs(is2 - is0)
    s = sum(c * (1 + (tau / (b + 1e-40)) ** 2) for c, b in zip((0.2, 0.5, 0.3), (is0, is1, is2)))
    return 1.0 / (1.0 + (s - 1.0) ** 2)


def theta_faces(q, m, d, gamma):
    """Per face of the periodic line (faces 0..L-1): the smallest theta of density and
    pressure over the positive (f-3 .. f+1) and negative (f+2 .. f-2) stencils."""
    _, _, rho, p = lf_split(q, m, d, gamma)
    ln = PeriodicLine(d, rho.shape)
    out = None
    for a in (rho, p):
        for offs in ((-3, -2, -1, 0, 1), (2, 1, 0, -1, -2)):
            t = theta_stencil(*[ln.at(a, c) for c in offs])
            out = t if out is None else np.minimum(out, t)
    return out
