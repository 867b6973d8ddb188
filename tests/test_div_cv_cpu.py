"""The division by cv = 1/(gamma-1) of uprim (src/uprim.f90) as two FP64
operations, fma(x, h, x*l) with h = RN(1/cv), l = RN(1/cv - h), which the
device uses when the odd part C of cv's significand is small
(walicxe2d_b200/csrc/w2d_phys.cuh: cv_split, div_cv).  The argument: x/cv
lies at least ulp/(2C) from every rounding midpoint, and the fma's one
rounding acts on a value within ~2^-104 |x/cv| of x/cv, so the result is
the correctly rounded x/cv (for |x| >= 2^-960; zeros and smaller x divide).

Checked here in exact rational arithmetic (Python's float / is IEEE
division): the fma's value x*h + RN(x*l) rounded once against x / cv, for
random x over many binades and for x built so that x/cv falls as near a
midpoint as it can (x = RN(cv * m), m a midpoint), for the reference's
cv = 1.5 (src/parameters.f90:39, gamma = (cv+1)/cv) and for 2.5, 3, 1000
and 2; and the eligibility rule on a cv whose odd part is large.
"""
import math
import random
from fractions import Fraction as F

import pytest


def split(cv):
    """cv_split of w2d_phys.cuh: (h, l) or None."""
    if not (cv > 0 and math.isfinite(cv)):
        return None
    m, e = math.frexp(cv)
    M = int(math.ldexp(m, 53))
    while M % 2 == 0:
        M //= 2
    if M >= 1 << 20:
        return None
    h = 1.0 / cv
    r = float(F(1) - F(cv) * F(h))          # exact: 1 - cv*h is a double
    assert F(r) == F(1) - F(cv) * F(h)
    return h, r / cv


def div_cv(x, h, l, cv):
    """div_cv of w2d_phys.cuh: the fma for |x| >= 2^-960, else the division."""
    if not abs(x) >= 2.0 ** -960:
        return x / cv
    return float(F(x) * F(h) + F(x * l))    # fma(x, h, RN(x*l)): one rounding


def midpoint_inputs(cv, rng, n):
    out = []
    for _ in range(n):
        q = math.ldexp(1.0 + rng.random(), rng.randint(-40, 40))
        half = math.ldexp(math.ulp(q), -1)
        m = F(q) + F(half)                   # a midpoint between doubles
        x = float(m * F(cv))                 # RN(cv * m)
        for d in (-1, 0, 1):                 # and its neighbours
            out.append(math.nextafter(x, math.inf) if d > 0 else (math.nextafter(x, -math.inf) if d < 0 else x))
    return out


@pytest.mark.parametrize("cv", [1.5, 2.5, 3.0, 1000.0, 2.0])
def test_two_op_division_is_correctly_rounded(cv):
    hl = split(cv)
    assert hl is not None, cv
    h, l = hl
    rng = random.Random(20261204)
    xs = [math.ldexp(rng.random() * 2 - 1, rng.randint(-300, 300)) for _ in range(20000)]
    xs += midpoint_inputs(cv, rng, 4000)
    xs += [0.0, -0.0, 1.0, -1.0, cv, 3.0, 1e-15, 2.0 ** -960]
    bad = [x for x in xs if div_cv(x, h, l, cv) != x / cv]
    assert not bad, bad[:5]
    # zeros keep their sign: they take the division (the fma would turn
    # -0 into +0 where l < 0, as for cv = 2.5 and 1000)
    assert math.copysign(1.0, div_cv(-0.0, h, l, cv)) == -1.0
    if l < 0:
        assert math.copysign(1.0, (-0.0 * h) + (-0.0 * l)) == 1.0


def test_split_refuses_a_cv_with_a_large_odd_part():
    assert split(1.5) is not None and split(2.5) is not None and split(1000.0) is not None
    assert split(1.0 / (1.3 - 1.0)) is None       # 3.333...: a full 53-bit odd significand
    assert split(1.0 / (5.0 / 3.0 - 1.0)) is None  # 1.4999999999999998, cv from gamma in doubles
    assert split(0.0) is None and split(-1.5) is None and split(math.inf) is None
