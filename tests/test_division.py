"""The branch-free quotient of the residual kernel's MUSCL limiter
(shared_cfd_b200/csrc/div_pos.cuh, used by the residual kernel), restated step by step in exact
rational arithmetic, each operation (a fused multiply-add included) rounded once
to nearest-even in the kernel's precision.  From reciprocal seeds up to 2^-21
off (the hardware's approximate reciprocal is good to about 2^-23), the
quotient is within one unit in the last place of a / b and equals the correctly
rounded quotient in nearly every case.  The limiter's quotients are
2 Du Dl / (Du^2 + Dl^2 + eps) with differences Du, Dl of every magnitude the
primitive field holds."""
from fractions import Fraction as Fr

import numpy as np
import pytest


def rnd(x, p):
    """x rounded to nearest-even with a p-bit significand (normal range)."""
    if x == 0:
        return Fr(0)
    s = -1 if x < 0 else 1
    x = abs(x)
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if Fr(2) ** e > x:
        e -= 1
    scale = Fr(2) ** (e - p + 1)
    m = x / scale
    n = m.numerator // m.denominator
    r = m - n
    if r > Fr(1, 2) or (r == Fr(1, 2) and n % 2 == 1):
        n += 1
    return s * n * scale


def ulp(x, p):
    x = abs(x)
    e = x.numerator.bit_length() - x.denominator.bit_length()
    if Fr(2) ** e > x:
        e -= 1
    return Fr(2) ** (e - p + 1)


def div_pos(a, b, y0, p):
    """the kernel's steps: FP64 (p = 53) a third-order, FP32 (p = 24) a
    second-order Newton-Raphson step on the reciprocal, then Markstein's
    remainder correction"""
    fma = lambda x, y, z: rnd(x * y + z, p)
    e = fma(-b, y0, Fr(1))
    y = fma(fma(e, e, e), y0, y0) if p == 53 else fma(e, y0, y0)
    q = rnd(a * y, p)
    return fma(fma(-b, q, a), y, q)


def limiter_operands(rng, n, p, eps):
    """(a, b) = (2 Du Dl, Du^2 + Dl^2 + eps), both rounded as the kernel rounds them"""
    out = []
    for _ in range(n):
        du = Fr(float(rng.choice([-1, 1]) * 10.0 ** rng.uniform(-20, 7)))
        dl = Fr(float(rng.choice([-1, 1]) * 10.0 ** rng.uniform(-20, 7)))
        if rng.random() < 0.5:  # smooth regions: Du and Dl of one magnitude
            dl = Fr(float(du) * rng.uniform(-3, 3))
        du, dl = rnd(du, p), rnd(dl, p)
        a = rnd(rnd(2 * du, p) * dl, p)
        b = rnd(rnd(rnd(du * du, p) + rnd(dl * dl, p), p) + eps, p)
        out.append((a, b))
    return out


@pytest.mark.parametrize("p,eps", [(53, Fr(1e-300)), (24, Fr(float(np.float32(1e-37))))])
def test_limiter_quotient_within_one_ulp(p, eps):
    rng = np.random.default_rng(5)
    ops = limiter_operands(rng, 1500, p, eps)
    # and plain positive denominators over a wide range
    for _ in range(500):
        a = rnd(Fr(float(rng.choice([-1, 1]) * 10.0 ** rng.uniform(-30, 30))), p)
        b = rnd(Fr(float(10.0 ** rng.uniform(-30, 30))), p)
        ops.append((a, b))
    exact_hits = 0
    for a, b in ops:
        delta = Fr(float(rng.uniform(-1, 1))) * Fr(1, 2 ** 21)
        y0 = rnd((1 / b) * (1 + delta), p)
        q = div_pos(a, b, y0, p)
        t = a / b
        if t == 0:
            assert q == 0
            exact_hits += 1
            continue
        assert abs(q - t) <= ulp(t, p), (float(a), float(b), float(q), float(t))
        exact_hits += q == rnd(t, p)
    assert exact_hits >= 0.99 * len(ops), exact_hits
