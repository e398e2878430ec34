"""Synthetic workloads with the shapes of the reference's benchmark configurations.

No dataset is involved: every state is generated from a formula.
  * taylor_green     -- block::initial_taylorgreen (src/block.cpp:683-690), periodic box
  * spherical_riemann-- rho, p = 1, 10 for r < 0.2 and 0.125, 0.1 outside, u = 0,
                        outlet (extrapolation) faces; the reference has no initialiser
                        for it, so the state is injected like its restart file
                        (src/block.cpp:785-816)
  * isotropic_turbulence + uneven_blocks -- decaying isotropic turbulence in a periodic
                        2 pi box cut into blocks of uneven sizes (seeded), injected the same way
  * shock_turbulence -- a Rankine-Hugoniot normal shock in that turbulence, inflow/outflow
                        in x, periodic y and z
  * boundary_layer   -- a supersonic boundary layer over a Gaussian bump on a tanh-stretched
                        mesh in uneven blocks, isothermal wall
Uniform boxes get analytic metrics (xi_x = 1/hx, jac = 1/(hx hy hz)); curvilinear
meshes go through nuc3d_b200.metrics (block::getJacobians).
"""
from __future__ import annotations

import math

import numpy as np

PERIODIC_NEIGHBOUR_FACE = (1, 0, 3, 2, 5, 4)


def uniform_metrics(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)) -> dict:
    nx, ny, nz = shape
    h = [(hi[d] - lo[d]) / n for d, n in enumerate(shape)]
    N = (nz, ny, nx)
    one = np.ones(N)
    zero = np.zeros(N)
    jac = one / (h[0] * h[1] * h[2])
    return {
        "jac": jac,
        "xi_xyz": np.stack([one / h[0], zero, zero]),
        "eta_xyz": np.stack([zero, one / h[1], zero]),
        "zeta_xyz": np.stack([zero, zero, one / h[2]]),
        "dxyz": np.stack([one * h[0], zero, zero, zero, one * h[1], zero, zero, zero, one * h[2]]),
    }


def centres(shape, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    nx, ny, nz = shape
    c = [lo[d] + (np.arange(n) + 0.5) * (hi[d] - lo[d]) / n for d, n in enumerate(shape)]
    Z, Y, X = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    return X, Y, Z


def prim_to_q(prim, jac, gamma):
    """U/J with the arithmetic of block::initialQ (src/block.cpp:554-563)."""
    rho, u, v, w, p = prim
    rhoe = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return np.stack([rho / jac, (rho * u) / jac, (rho * v) / jac, (rho * w) / jac, rhoe / jac])


def unit_box_nodes(shape):
    """Node coordinates (x, y, z), each (nz+1, ny+1, nx+1), of the unit box: i/nx, j/ny,
    k/nz, the mesh the reference reads for the shock-dominated workload.  Metrics taken from
    them by block::getJacobians (nuc3d_block_set_nodes) are the reference's own, bit for bit;
    the analytic uniform_metrics differ from those in the last bits."""
    xs = [np.arange(n + 1, dtype=np.float64) / n for n in shape]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    return X, Y, Z


def spherical_riemann(shape, gamma=1.4, radius=0.2):
    X, Y, Z = centres(shape)
    r2 = (X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2
    inside = r2 < radius * radius
    rho = np.where(inside, 1.0, 0.125)
    p = np.where(inside, 10.0, 0.1)
    zero = np.zeros_like(rho)
    m = uniform_metrics(shape)
    return prim_to_q(np.stack([rho, zero, zero, zero, p]), m["jac"], gamma), m


def gaussian_pulse(shape, gamma=1.4, amp=0.5, width=0.08):
    """Smooth isentropic pressure pulse at rest in the unit box: rho = 1 + amp g,
    p = rho^gamma / gamma, g = exp(-r^2 / width^2) about the centre (sound speed 1 in the
    far field).  A case the compact schemes resolve without the oscillations a
    discontinuity gives them."""
    X, Y, Z = centres(shape)
    g = np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2 + (Z - 0.5) ** 2) / (width * width))
    rho = 1.0 + amp * g
    p = rho ** gamma / gamma
    zero = np.zeros_like(rho)
    m = uniform_metrics(shape)
    return prim_to_q(np.stack([rho, zero, zero, zero, p]), m["jac"], gamma), m


def taylor_green(shape, gamma=1.4, mach=0.1):
    lo, hi = (0.0,) * 3, (2.0 * math.pi,) * 3
    X, Y, Z = centres(shape, lo, hi)
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    rho = np.ones_like(u)
    p = 1.0 / (gamma * mach * mach) + ((np.cos(2.0 * Z) + 2.0) * (np.cos(2.0 * X) + np.cos(2.0 * Y)) - 2.0) / 16.0
    m = uniform_metrics(shape, lo, hi)
    return prim_to_q(np.stack([rho, u, v, w, p]), m["jac"], gamma), m


def outlet_faces():
    return [-1] * 6, [1] * 6


def periodic_faces(block=0):
    return [block] * 6, list(PERIODIC_NEIGHBOUR_FACE)


def isotropic_turbulence(shape, seed=0, k0=4.0, mt=0.6, gamma=1.4, re_lambda=100.0):
    """Seeded random-phase solenoidal velocity on the periodic [0, 2 pi]^3 box of
    shape = (nx, ny, nz) cells, energy spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), rho = T = 1.

    Nondimensionalised as the reference (T = gamma Ma^2 p / rho): with the reference Mach
    number Ma = mt and the velocity scaled to rms |u| = 1 the sound speed is 1/mt, so the
    turbulent Mach number is mt.  Returns (prim (5, nz, ny, nx), reynolds) where reynolds
    is the reference's Reynolds number that gives Taylor-scale Reynolds number re_lambda
    (mu(T = 1) = 1/Re under Sutherland's law)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    kz = np.fft.fftfreq(nz, 1.0 / nz)[:, None, None]
    ky = np.fft.fftfreq(ny, 1.0 / ny)[None, :, None]
    kx = np.fft.fftfreq(nx, 1.0 / nx)[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k = np.sqrt(k2)
    amp = np.where(k > 0, np.sqrt(k ** 4 * np.exp(-2.0 * (k / k0) ** 2) / np.maximum(k2, 1.0)), 0.0)
    # no Nyquist modes: their real part has no conjugate partner to stay solenoidal with
    amp = np.where((np.abs(kx) == nx // 2) | (np.abs(ky) == ny // 2) | (np.abs(kz) == nz // 2), 0.0, amp)
    comps = []
    for _ in range(3):
        ph = rng.uniform(0.0, 2.0 * np.pi, k.shape)
        comps.append(amp * (rng.standard_normal(k.shape)) * np.exp(1j * ph))
    # solenoidal projection: u_hat - k (k . u_hat) / k^2
    kd = (kx * comps[0] + ky * comps[1] + kz * comps[2]) / np.maximum(k2, 1.0)
    uh = [comps[0] - kx * kd, comps[1] - ky * kd, comps[2] - kz * kd]
    vel = [np.real(np.fft.ifftn(c)) for c in uh]
    scale = 1.0 / np.sqrt(np.mean(vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2))
    u, v, w = (scale * a for a in vel)
    # Taylor scale from the spectral derivative of u along x
    dudx = np.real(np.fft.ifftn(1j * kx * np.fft.fftn(u)))
    urms = np.sqrt(np.mean(u * u))
    lam = urms / np.sqrt(np.mean(dudx * dudx))
    rho = np.ones_like(u)
    p = rho / (gamma * mt * mt)
    return np.stack([rho, u, v, w, p]), re_lambda / (urms * lam)


def normal_shock(m1, gamma=1.4):
    """Rankine-Hugoniot jumps of a normal shock of upstream Mach number m1: (rho2/rho1,
    u2/u1, p2/p1)."""
    r = (gamma + 1.0) * m1 * m1 / ((gamma - 1.0) * m1 * m1 + 2.0)
    return r, 1.0 / r, 1.0 + 2.0 * gamma / (gamma + 1.0) * (m1 * m1 - 1.0)


def shock_turbulence(shape=(512, 256, 256), m1=1.5, x_shock=0.5 * math.pi, seed=7, mt=0.6,
                     gamma=1.4, re_lambda=100.0):
    """A Mach m1 normal shock at x = x_shock in the decaying-turbulence field of the
    24-block workload: the box [0, 2 pi nx/ny] x [0, 2 pi]^2 with uniform spacing 2 pi/ny,
    periodic in y and z, inflow through x = 0 and outflow through the far x face.

    Nondimensionalised as the reference (T = gamma Ma^2 p / rho) with Ma = mt: upstream
    rho = T = 1, so the sound speed is 1/mt and the mean velocity m1/mt along x; downstream
    the Rankine-Hugoniot state.  The solenoidal fluctuation of isotropic_turbulence (rms
    |u| = 1, turbulent Mach number mt, its 2 pi period repeated along x) is added on both
    sides.  Returns (prim (5, nz, ny, nx), reynolds, inlet (rho, u, v, w, p) of the x- face,
    node coordinates (x, y, z))."""
    nx, ny, nz = shape
    h = 2.0 * math.pi / ny
    turb, re = isotropic_turbulence((ny, ny, nz), seed=seed, mt=mt, gamma=gamma, re_lambda=re_lambda)
    reps = -(-nx // ny)
    fl = np.concatenate([turb[:, :, :, :]] * reps, axis=3)[:, :, :, :nx]
    xc = (np.arange(nx) + 0.5) * h
    up = xc < x_shock
    rr, ur, pr = normal_shock(m1, gamma)
    rho1, p1 = 1.0, 1.0 / (gamma * mt * mt)
    u1 = m1 / mt
    rho = np.where(up, rho1, rho1 * rr)[None, None, :] * np.ones((nz, ny, 1))
    umean = np.where(up, u1, u1 * ur)[None, None, :]
    p = np.where(up, p1, p1 * pr)[None, None, :] * np.ones((nz, ny, 1))
    prim = np.stack([rho, umean + fl[1], fl[2], fl[3], p])
    xs = np.arange(nx + 1) * h
    ys = np.arange(ny + 1) * h
    zs = np.arange(nz + 1) * h
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    return prim, re, (rho1, u1, 0.0, 0.0, p1), (X, Y, Z)


def shock_faces(block=0):
    """BC_Topo of the shock-turbulence block: inlet on x-, outlet on x+, periodic y and z."""
    return [-1, -1, block, block, block, block], [0, 1, 3, 2, 5, 4]


def shock_position(rho, h):
    """x of the shock: where the density averaged over y and z first reaches the mean of
    its upstream (first column) and downstream (last column) values, linearly interpolated
    between cell centres."""
    prof = rho.mean(axis=(0, 1))
    mid = 0.5 * (prof[0] + prof[-1])
    i = int(np.argmax(prof >= mid))
    if i == 0:
        return 0.5 * h
    t = (mid - prof[i - 1]) / (prof[i] - prof[i - 1])
    return (i - 0.5 + t) * h


def split_sizes(total, parts, seed, quantum=4, spread=0.25):
    """`parts` uneven extents (multiples of `quantum`) summing to `total`, drawn with a
    fixed seed within +-spread of the even split."""
    rng = np.random.default_rng(seed)
    base = total / parts
    while True:
        w = base * (1.0 + spread * rng.uniform(-1.0, 1.0, parts))
        n = [max(quantum, int(round(x / quantum)) * quantum) for x in w[:-1]]
        last = total - sum(n)
        if last >= quantum and last % quantum == 0:
            return n + [last]


def boundary_layer(shape=(1024, 256, 128), nblocks=(4, 2, 2), seed=5, mach=2.25, t_wall=1.9,
                   re_delta=1581.0, lengths=(32.0, 8.0, 4.0), bump=(12.0, 0.5, 2.0),
                   stretch=2.5, gamma=1.4):
    """Supersonic flat-plate boundary layer over a Gaussian roughness bump, cut into
    nblocks (x, y, z) uneven blocks.

    Lengths in units of the inflow boundary-layer thickness delta; the bump y_w(x) =
    h exp(-((x - x_b)/w)^2) with (x_b, h, w) = bump, h = 0.5 delta, w = 2 delta.  Nodes:
    x and z uniform; y from the local wall to the top, clustered at the wall by tanh
    stretching, y = y_w + (Ly - y_w) (1 - tanh(b (1 - s)) / tanh(b)), s uniform in [0, 1].
    Nondimensionalised as the reference (T = gamma Ma^2 p / rho) with the free stream
    rho = T = u = 1, Ma = mach; Reynolds number per delta re_delta (Re_x = 1e5 at the
    inflow with the Blasius thickness delta = 5 x / sqrt(Re_x)).  Initial state: a tanh
    velocity profile u = tanh(3 d / delta) in the wall distance d, the Crocco-Busemann
    temperature between the isothermal wall T_w = t_wall and the free stream (recovery
    factor 0.89), uniform pressure.  Faces: inlet (free stream) on x-, outlet on x+,
    isothermal wall on y-, outlet on y+, periodic z.
    Returns (blocks, types, ids, values, params): blocks a list of dicts with 'shape',
    'lo' (cell offsets), 'nodes' (x, y, z), 'prim' (5, nz, ny, nx); types/ids/values per
    block as nuc3d_block_add takes them; params the PhysModel values."""
    nx, ny, nz = shape
    parts = [split_sizes(shape[d], nblocks[d], seed + d) for d in range(3)]
    Lx, Ly, Lz = lengths
    xb, hb, wb = bump
    xs = np.arange(nx + 1) * (Lx / nx)
    zs = np.arange(nz + 1) * (Lz / nz)
    sgrid = np.arange(ny + 1) / ny
    yw = hb * np.exp(-((xs - xb) / wb) ** 2)
    fr = 1.0 - np.tanh(stretch * (1.0 - sgrid)) / np.tanh(stretch)
    Yn = yw[None, :] + (Ly - yw[None, :]) * fr[:, None]          # (ny+1, nx+1)
    p_inf = 1.0 / (gamma * mach * mach)
    t_rec = 1.0 + 0.89 * 0.5 * (gamma - 1.0) * mach * mach
    types, ids, values = [], [], []
    na, nb_, nc = nblocks
    idx = lambda a, b, c: a + na * (b + nb_ * c)  # noqa: E731
    off = [np.concatenate([[0], np.cumsum(p)]) for p in parts]
    inlet = [1.0, 1.0, 0.0, 0.0, p_inf]
    blocks = []
    for c in range(nc):
        for b in range(nb_):
            for a in range(na):
                lo = (int(off[0][a]), int(off[1][b]), int(off[2][c]))
                n = (parts[0][a], parts[1][b], parts[2][c])
                xi = xs[lo[0]:lo[0] + n[0] + 1]
                zi = zs[lo[2]:lo[2] + n[2] + 1]
                yi = Yn[lo[1]:lo[1] + n[1] + 1, lo[0]:lo[0] + n[0] + 1]
                X = np.broadcast_to(xi[None, None, :], (n[2] + 1, n[1] + 1, n[0] + 1)).copy()
                Y = np.broadcast_to(yi[None, :, :], (n[2] + 1, n[1] + 1, n[0] + 1)).copy()
                Z = np.broadcast_to(zi[:, None, None], (n[2] + 1, n[1] + 1, n[0] + 1)).copy()
                # cell centres (averages of the 8 nodes) and their wall distance
                cen = lambda A: 0.125 * (A[:-1, :-1, :-1] + A[1:, :-1, :-1] + A[:-1, 1:, :-1] + A[:-1, :-1, 1:]
                                         + A[1:, 1:, :-1] + A[1:, :-1, 1:] + A[:-1, 1:, 1:] + A[1:, 1:, 1:])  # noqa: E731
                xc, yc = cen(X), cen(Y)
                dist = yc - hb * np.exp(-((xc - xb) / wb) ** 2)
                u = np.tanh(3.0 * np.maximum(dist, 0.0))
                T = t_wall + (t_rec - t_wall) * u + (1.0 - t_rec) * u * u
                p = np.full_like(u, p_inf)
                rho = p * gamma * mach * mach / T
                zero = np.zeros_like(u)
                blocks.append(dict(shape=n, lo=lo, nodes=(X, Y, Z), prim=np.stack([rho, u, zero, zero, p])))
                t, i, v = [], [], np.zeros((6, 5))
                pos = (a, b, c)
                for f in range(6):
                    d, side = f // 2, f % 2
                    q = list(pos)
                    q[d] += 1 if side else -1
                    if d == 2:  # periodic spanwise
                        q[2] %= nc
                        t.append(idx(*q)); i.append(f ^ 1)
                    elif 0 <= q[d] < nblocks[d]:
                        t.append(idx(*q)); i.append(f ^ 1)
                    elif f == 0:
                        t.append(-1); i.append(0); v[0] = inlet
                    elif f == 2:
                        t.append(-1); i.append(2)
                    else:
                        t.append(-1); i.append(1)
                types.append(t); ids.append(i); values.append(v)
    params = {"Reynolds": re_delta, "Mach": mach, "Pt": 0.72, "Gamma": gamma, "T_ref": 110.4,
              "T_inf": 288.0, "T_wall": t_wall}
    return blocks, types, ids, values, params


def uneven_blocks(nblocks=(2, 3, 4), sizes=(48, 64, 96, 128, 160), seed=0):
    """Per-axis block sizes of a tensor-product partition, drawn with a fixed seed
    (neighbouring faces match, as the reference's buffers require:
    src/bufferData.cpp:16-47).  Returns [sizes along x, along y, along z]."""
    rng = np.random.default_rng(seed)
    return [[int(s) for s in rng.choice(sizes, size=n)] for n in nblocks]


def block_topology(parts):
    """Blocks of a periodic tensor-product partition, x fastest: for block (a, b, c) the
    BC_Topo face types (neighbour block index) and ids (neighbour face)."""
    na, nb, nc = (len(p) for p in parts)
    idx = lambda a, b, c: a + na * (b + nb * c)  # noqa: E731
    types, ids = [], []
    for c in range(nc):
        for b in range(nb):
            for a in range(na):
                pos, n = [a, b, c], [na, nb, nc]
                t = []
                for f in range(6):
                    d, side = f // 2, f % 2
                    q = list(pos)
                    q[d] = (q[d] + (1 if side else -1)) % n[d]
                    t.append(idx(*q))
                types.append(t)
                ids.append(list(PERIODIC_NEIGHBOUR_FACE))
    return types, ids
