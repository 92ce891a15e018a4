"""The elementary functions of the FP64 parity build (gx_math.h).

The CUDA library's FP64 parity variant and the oracle's parity build compile
the same header, so that both round alike; here its error is bounded on the
CPU against the C library (whose log, exp, sin, cos are within an ulp of the
true value or correctly rounded) and against high-precision decimal values,
over the argument ranges the transport uses.  The GPU tests check that the
device compiles it to the same bits (tests/test_gpu_parity_transport.py).
"""
from decimal import Decimal, getcontext

import numpy as np
import pytest

from oracle_ctypes import Oracle

# largest difference from the C library, in ulps of the C library's value
BOUND_VS_LIBM = {"log": 1, "exp": 1, "pow": 1, "sin": 1, "cos": 1, "expm1": 2, "log1p": 1}
# largest error against the true value (decimal, 50 digits), in ulps
BOUND_TRUE = {"log": 1.0, "exp": 1.0, "pow": 1.5, "expm1": 2.0, "log1p": 1.0}


@pytest.fixture(scope="module")
def orc():
    return Oracle()


def _ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


def _args(name, n, rng):
    if name == "log":
        return [np.exp(rng.uniform(-700, 700, n)), 1 + rng.uniform(-0.3, 0.42, n), np.exp(rng.uniform(-740, -705, 500))]
    if name == "exp":
        return [rng.uniform(-745, 709, n), rng.uniform(-1, 1, n), rng.uniform(-1e-8, 1e-8, n)]
    if name in ("sin", "cos"):
        return [rng.uniform(0, 2 * np.pi, n), rng.uniform(-1e3, 1e3, n), rng.uniform(-1e6, 1e6, n)]
    if name == "expm1":
        return [rng.uniform(-40, 40, n), rng.uniform(-0.5, 0.5, n), rng.uniform(-1e-6, 1e-6, n)]
    if name == "log1p":
        return [rng.uniform(-0.999, 1e3, n), rng.uniform(-1e-6, 1e-6, n), rng.uniform(-0.5, 0.5, n)]
    raise KeyError(name)


@pytest.mark.parametrize("name", ["log", "exp", "sin", "cos", "expm1", "log1p"])
def test_against_the_c_library(orc, name):
    rng = np.random.default_rng(11)
    for x in _args(name, 100000, rng):
        got, want = orc.math_eval(name, x), orc.math_eval(name, x, libm=True)
        assert np.all(np.isfinite(got))
        assert _ulps(got, want).max() <= BOUND_VS_LIBM[name], name


def test_pow_against_the_c_library(orc):
    rng = np.random.default_rng(12)
    n = 100000
    # the transport's uses: u^0.333333 for u in (0, 1), Z^(1/3), x^(1/3) for x in [1, 3];
    # and a wide sweep
    x = np.concatenate([rng.uniform(0, 1, n), rng.uniform(1, 100, n), np.exp(rng.uniform(-700, 700, n))])
    y = np.concatenate([np.full(n, 0.333333), np.full(n, 1 / 3.0), rng.uniform(-1, 1, n)])
    got, want = orc.math_eval("pow", x, y), orc.math_eval("pow", x, y, libm=True)
    assert _ulps(got, want).max() <= BOUND_VS_LIBM["pow"]


def test_special_values(orc):
    inf, nan = np.inf, np.nan
    x = np.array([0.0, 1.0, inf, -1.0, nan])
    got = orc.math_eval("log", x)
    assert got[0] == -inf and got[1] == 0.0 and got[2] == inf and np.isnan(got[3]) and np.isnan(got[4])
    got = orc.math_eval("exp", np.array([0.0, 710.0, -746.0, -inf, nan]))
    assert got[0] == 1.0 and got[1] == inf and got[2] == 0.0 and got[3] == 0.0 and np.isnan(got[4])
    got = orc.math_eval("log1p", np.array([0.0, -1.0, -2.0, 1e-300]))
    assert got[0] == 0.0 and got[1] == -inf and np.isnan(got[2]) and got[3] == 1e-300
    got = orc.math_eval("expm1", np.array([0.0, -50.0, 1e-300]))
    assert got[0] == 0.0 and got[1] == -1.0 and got[2] == 1e-300
    got = orc.math_eval("pow", np.array([0.0, 2.0, 1.0, 8.0]), np.array([2.0, 0.0, 1e10, 1 / 3.0]))
    assert got[0] == 0.0 and got[1] == 1.0 and got[2] == 1.0 and abs(got[3] - 2.0) <= 4.5e-16
    s, c = orc.math_eval("sin", np.array([0.0, np.pi / 2])), orc.math_eval("cos", np.array([0.0, np.pi]))
    assert s[0] == 0.0 and s[1] == 1.0 and c[0] == 1.0 and c[1] == -1.0


@pytest.mark.parametrize("name", ["log", "exp", "expm1", "log1p", "pow"])
def test_against_high_precision_values(orc, name):
    getcontext().prec = 50
    rng = np.random.default_rng(13)
    m = 1500
    y = None
    if name == "log":
        x = np.concatenate([np.exp(rng.uniform(-700, 700, m)), 1 + rng.uniform(-0.3, 0.42, m)])
    elif name == "exp":
        x = rng.uniform(-700, 700, m)
    elif name == "expm1":
        x = np.concatenate([rng.uniform(-40, 40, m), rng.uniform(-0.5, 0.5, m), rng.uniform(-1e-5, 1e-5, m)])
    elif name == "log1p":
        x = np.concatenate([rng.uniform(-0.999, 1e3, m), rng.uniform(-0.5, 0.5, m)])
    else:
        x = np.concatenate([rng.uniform(0, 1, m), rng.uniform(1, 100, m)])
        y = np.concatenate([np.full(m, 0.333333), rng.uniform(-3, 3, m)])
    got = orc.math_eval(name, x, y)
    worst = 0.0
    for i in range(len(x)):
        X = Decimal(float(x[i]))
        t = {"log": lambda: X.ln(), "exp": lambda: X.exp(), "expm1": lambda: X.exp() - 1,
             "log1p": lambda: (1 + X).ln(), "pow": lambda: (Decimal(float(y[i])) * X.ln()).exp()}[name]()
        worst = max(worst, float(abs(Decimal(float(got[i])) - t) / Decimal(float(np.spacing(abs(float(t)))))))
    assert worst <= BOUND_TRUE[name], (name, worst)
