"""The FP64 form divides by 6 in WENO5 (reconstruction.cpp:117-119) as
div_rcp(a, 6, RN(1/6)) = RN(q + (a - 6 q) y) with q = RN(a y): three FMA-unit
operations instead of an IEEE division. Markstein's theorem says the result is
the IEEE quotient bit for bit; this checks the method itself in exact rational
arithmetic (the device's FMA rounds exactly once, as Fraction -> float does
here) against Python's IEEE division, on random operands over 120 binades and
on operands next to multiples of the divisor. The GPU parity tests then check
the kernels that use it."""
import math
import random
from fractions import Fraction

import pytest


def div_rcp(a: float, b: float, y: float) -> float:
    q = float(Fraction(a) * Fraction(y))          # RN(a * y)
    r = Fraction(a) - Fraction(b) * Fraction(q)   # one FMA: exact by the theorem
    assert float(r) == r
    return float(Fraction(q) + r * Fraction(y))   # RN(q + r * y), one FMA


@pytest.mark.parametrize("b", [6.0, 2.8, 120960.0])
def test_division_by_a_precomputed_reciprocal_is_the_ieee_quotient(b):
    y = 1.0 / b
    rng = random.Random(7)
    for _ in range(20000):
        a = rng.uniform(1.0, 2.0) * 2.0 ** rng.randint(-60, 60) * rng.choice((1.0, -1.0))
        assert div_rcp(a, b, y) == a / b, a
    for k in range(1, 3000):
        for a in (k * b, math.nextafter(k * b, 0.0), math.nextafter(k * b, math.inf)):
            assert div_rcp(a, b, y) == a / b, a
    assert div_rcp(0.0, b, y) == 0.0
