"""The branch-free FP64 exp, tanh and square roots of csrc/fastmath.cuh.

CPU: the exponential's operations (Cody-Waite reduction against ln 2, the
degree-13 Taylor polynomial in Estrin form, the exponent-field scale) are
emulated with exact fused multiply-adds, with the constants read from the
header, and held against libm: within 1 ulp.  GPU: the device functions
(hdnnp_debug_math) against numpy's libm results: exp and 1/sqrt within 2 ulp,
sqrt within 1 ulp, tanh on [0, 1] within 6e-16 absolute (the subtraction
1 - e^(-2u) keeps the absolute, not the relative error of e^(-2u); the
cutoff function tanh^3 and its derivative vanish as u -> 0).  These replace the
library calls of the reference's intrinsics exp, tanh and sqrt
(symmetryFunctions.f90:201-327) in the symmetry-function kernels.
"""
import math
import os
import re
import struct
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "high-dimensional-neural-network-potential_b200", "csrc", "fastmath.cuh")


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _exp_constants():
    src = open(HEADER).read()
    body = src[src.index("double exp_clamped(double x)"):]
    body = body[: body.index("\n}\n")]
    named = dict(re.findall(r"constexpr double (\w+) = ([0-9.eE+-]+);", body))
    pairs = re.findall(r"fma\(([0-9.eE+-]+), r, ([0-9.eE+-]+)\)", body)
    return {k: float(v) for k, v in named.items()}, [(float(a), float(b)) for a, b in pairs]


def _exp_emulated(x, K, Q):
    x = min(max(x, -708.0), 709.0)
    t = _fma(x, K["kLog2e"], K["kShift"])
    k = struct.unpack("<q", struct.pack("<d", t))[0] & 0xFFFFFFFF
    k = k - (1 << 32) if k >= (1 << 31) else k
    kd = t - K["kShift"]
    r = _fma(kd, -K["kLn2Hi"], x)
    r = _fma(kd, -K["kLn2Lo"], r)
    r2 = r * r
    r4 = r2 * r2
    r8 = r4 * r4
    q = [r] + [_fma(a, r, b) for a, b in Q]  # q0 .. q6
    s0 = _fma(q[1], r2, q[0])
    s1 = _fma(q[3], r2, q[2])
    s2 = _fma(q[5], r2, q[4])
    t0 = _fma(s1, r4, s0)
    t1 = _fma(q[6], r4, s2)
    p = 1.0 + _fma(t1, r8, t0)
    return p * math.ldexp(1.0, k)


def test_exp_emulation_within_one_ulp():
    K, Q = _exp_constants()
    assert set(K) == {"kLog2e", "kLn2Hi", "kLn2Lo", "kShift"} and len(Q) == 6
    # the coefficients are 1/n! for n = 2..13
    assert all(abs(b - 1 / math.factorial(2 * i + 2)) <= 1e-16 / math.factorial(2 * i + 2) for i, (a, b) in enumerate(Q))
    rng = np.random.default_rng(7)
    xs = np.concatenate([-rng.random(600) * 5.0, -rng.random(200) * 700.0, rng.random(100) * 50.0, [0.0, -1e-300, -708.0]])
    worst = 0.0
    for x in xs:
        ref = math.exp(float(x))
        worst = max(worst, abs(_exp_emulated(float(x), K, Q) - ref) / math.ulp(ref))
    assert worst <= 1.0, worst


@pytest.mark.gpu
def test_device_functions_against_libm(pkg):
    from hdnnp_b200 import engine

    rng = np.random.default_rng(11)
    # exp: the symmetry functions' arguments -eta R (R up to 3 rc^2) and wide ranges
    x = np.concatenate([-rng.random(20000) * 5.0, -rng.random(20000) * 700.0, rng.random(2000) * 700.0, [0.0, -708.0]])
    y = engine.debug_math(0, x)
    ulp = np.abs(y - np.exp(x)) / np.spacing(np.exp(x))
    assert ulp.max() <= 2.0, ulp.max()
    # tanh of u = 1 - r/rc in [0, 1]
    u = np.concatenate([rng.random(40000), np.linspace(0.0, 1.0, 1001), [1e-12, 1e-6]])
    t = engine.debug_math(1, u)
    assert np.abs(t - np.tanh(u)).max() <= 6e-16
    big = u > 0.2
    assert (np.abs(t[big] - np.tanh(u[big])) / np.tanh(u[big])).max() <= 3e-15
    # square roots of squared distances (0 included: sqrt 0 = 0)
    r2 = np.concatenate([rng.random(40000) * 1000.0, rng.random(2000) * 1e-6, [0.0, 144.0]])
    s = engine.debug_math(2, r2)
    assert np.all(np.abs(s - np.sqrt(r2)) <= np.spacing(np.sqrt(r2)))
    pos = r2 > 0
    ir = engine.debug_math(3, r2[pos])
    ref = 1.0 / np.sqrt(r2[pos])
    assert (np.abs(ir - ref) / np.spacing(ref)).max() <= 2.0
    # bad selector
    with pytest.raises(engine.HdnnpError):
        engine.debug_math(7, x[:4])
