"""The energy reset's pow(rho, gamma) (src/physicsModel.cpp:329) in the oracle build.

The oracle and the GPU evaluate it with the double-double method of oracle/cr_pow.h
(its CUDA twin is cr_pow in physics.cuh); the result must be the correctly rounded x^y,
checked here against 200-bit arithmetic (mpmath), including where glibc's pow is not
correctly rounded."""
import math

import numpy as np
import pytest

from oracle import oracle as O


def test_cr_pow_correctly_rounded():
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    f = O.cr_pow
    rng = np.random.default_rng(11)
    xs = np.concatenate([rng.uniform(1e-3, 10.0, 3000), 10.0 ** rng.uniform(-30, 30, 2000)])
    ys = np.where(np.arange(xs.size) % 2 == 0, 1.4, rng.uniform(-5.0, 5.0, xs.size))
    libm_wrong = 0
    for x, y in zip(xs.tolist(), ys.tolist()):
        exact = float(mpmath.power(mpmath.mpf(x), mpmath.mpf(y)))
        assert f(x, y) == exact, (x, y, f(x, y), exact)
        libm_wrong += math.pow(x, y) != exact
    # the densities of the flows here, at gamma = 1.4
    for x in (0.125, 1.0, 10.0, 0.5, 3.7):
        assert f(x, 1.4) == float(mpmath.power(mpmath.mpf(x), mpmath.mpf(1.4)))
    assert f(1.0, 1.4) == 1.0 and f(4.0, 0.5) == 2.0
    print(f"glibc pow not correctly rounded on {libm_wrong} of {xs.size} samples")
