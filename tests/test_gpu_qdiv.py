"""Accuracy of the throughput build's division against IEEE division on the GPU.

The fast build divides with a reciprocal seed, one Newton-Raphson step and a
residual-corrected quotient (qdiv in physics.cuh).  On operands spanning the range
the WENO weights, flux splits and con2prim produce (|a|, |b| in 1e-150 .. 1e150,
both signs) it must agree with IEEE division to within one unit in the last place.
"""
import ctypes

import numpy as np
import pytest

from nuc3d_b200 import _LIB_PATH


@pytest.mark.gpu
def test_qdiv_within_one_ulp_of_ieee():
    lib = ctypes.CDLL(str(_LIB_PATH.with_name("libnuc3d_probe.so")))
    P = ctypes.POINTER(ctypes.c_double)
    lib.nuc3d_probe_qdiv.restype = ctypes.c_int
    lib.nuc3d_probe_qdiv.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_longlong]
    rng = np.random.default_rng(7)
    n = 1 << 22
    a = rng.uniform(1.0, 2.0, n) * 10.0 ** rng.uniform(-150, 150, n) * rng.choice([-1.0, 1.0], n)
    b = rng.uniform(1.0, 2.0, n) * 10.0 ** rng.uniform(-150, 150, n) * rng.choice([-1.0, 1.0], n)
    a[:4], b[:4] = (0.0, 1.0, -3.0, 7.0), (1.0, 3.0, 3.0, 7.0)
    qf, qi = np.empty(n), np.empty(n)
    ptr = lambda x: x.ctypes.data_as(P)  # noqa: E731
    assert lib.nuc3d_probe_qdiv(0, ptr(a), ptr(b), ptr(qf), ptr(qi), n) == 0
    assert np.array_equal(qi, a / b)  # the device's IEEE quotient is the host's
    ok = np.isfinite(qi) & (np.abs(qi) > np.finfo(np.float64).tiny)
    assert ok.mean() > 0.99
    ulp = np.abs(qf[ok].view(np.int64) - qi[ok].view(np.int64))
    assert int(ulp.max()) <= 1, int(ulp.max())
    assert np.mean(ulp == 0) > 0.99, np.mean(ulp == 0)
    assert qf[0] == 0.0 and qf[1] == 1.0 / 3.0 and qf[3] == 1.0


@pytest.mark.gpu
def test_cr_pow_bits_equal_the_oracle():
    """The energy reset's double-double pow (cr_pow in physics.cuh) returns on the GPU the
    bits the oracle's C evaluation of the same operations returns (oracle/cr_pow.h)."""
    from oracle import oracle as O
    lib = ctypes.CDLL(str(_LIB_PATH.with_name("libnuc3d_probe.so")))
    P = ctypes.POINTER(ctypes.c_double)
    lib.nuc3d_probe_crpow.restype = ctypes.c_int
    lib.nuc3d_probe_crpow.argtypes = [ctypes.c_int, P, P, P, ctypes.c_longlong]
    rng = np.random.default_rng(5)
    n = 20000
    x = np.concatenate([rng.uniform(1e-3, 10.0, n // 2), 10.0 ** rng.uniform(-60, 60, n // 2)])
    y = np.where(np.arange(n) % 2 == 0, 1.4, rng.uniform(-4.0, 4.0, n))
    r = np.empty(n)
    ptr = lambda a: a.ctypes.data_as(P)  # noqa: E731
    assert lib.nuc3d_probe_crpow(0, ptr(x), ptr(y), ptr(r), n) == 0
    want = np.array([O.cr_pow(float(a), float(b)) for a, b in zip(x, y)])
    assert np.array_equal(r.view(np.int64), want.view(np.int64)), int(np.sum(r != want))
