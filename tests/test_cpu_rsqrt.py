"""The device's FP64 reciprocal square roots (kemcu_device.cuh: rsqrt2_fast, rsqrt2_acc),
restated in Python with exactly rounded fused multiply-adds, from hardware estimates with the
largest relative error the refinement is designed for (2^-22), checked against the exactly
rounded 1/sqrt(x): the MIXED form within 1e-13 relative, the FP64 form within 1 ulp."""

import math
from fractions import Fraction

import numpy as np


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def rsqrt2_fast(x, y0):
    return y0 * fma(-(x * y0), y0, 3.0)


def rsqrt2_acc(x, y0):
    z = rsqrt2_fast(x, y0)
    e4 = fma(-(x * z), z, 4.0)
    return fma(0.125 * z, e4, z)


def exact_rsqrt(x):
    # 1/sqrt(x) to well beyond double precision (integer square root of a scaled numerator)
    f = Fraction(x)
    scale = 1 << 400
    r = math.isqrt((f.denominator * scale * scale) // f.numerator)
    return Fraction(r, scale)


def test_refined_reciprocal_square_roots():
    rng = np.random.default_rng(3)
    xs = np.exp(rng.uniform(np.log(1e-6), np.log(1e4), 400))  # squared distances in m^2
    worst_fast = worst_acc_ulp = 0.0
    for x in xs:
        x = float(x)
        ex = exact_rsqrt(x)
        for d in (-2.0 ** -22, 2.0 ** -22, float(rng.uniform(-2.0 ** -22, 2.0 ** -22))):
            y0 = float(1.0 / math.sqrt(x) * (1.0 + d))
            f = rsqrt2_fast(x, y0) * 0.5
            a = rsqrt2_acc(x, y0) * 0.5
            worst_fast = max(worst_fast, abs(float((Fraction(f) - ex) / ex)))
            worst_acc_ulp = max(worst_acc_ulp, abs(float(Fraction(a) - ex)) / math.ulp(float(ex)))
    assert worst_fast < 1e-13, worst_fast
    assert worst_acc_ulp <= 1.0, worst_acc_ulp
