"""Sutherland's law needs T^1.5 (field_structures.h:94-105, std::pow). The
FP64 form computes it as pow_1p5 (ns3d_device.cuh): s = RN(sqrt T),
r = T - s^2 (exact, one FMA), p = RN(T s), e = T s - p (exact, one FMA),
result RN(p + RN(e + RN(0.5 RN(r s)))). This checks the method in
exact rational arithmetic (each device operation rounds once, as
Fraction -> float does here) against the correctly rounded T^1.5 from
80-digit decimal arithmetic, and measures how often the host libm's pow (the
reference's) agrees with it."""
import math
import random
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 80


def rn(x: Fraction) -> float:
    return float(x)


def pow_1p5(T: float) -> float:
    s = math.sqrt(T)                                  # IEEE sqrt
    r = rn(Fraction(T) - Fraction(s) * Fraction(s))   # fma(-s, s, T)
    assert Fraction(r) == Fraction(T) - Fraction(s) ** 2  # exact residual
    p = T * s
    e = rn(Fraction(T) * Fraction(s) - Fraction(p))   # fma(T, s, -p)
    assert Fraction(e) == Fraction(T) * Fraction(s) - Fraction(p)
    return p + (e + 0.5 * (r * s))


def cr_pow_1p5(T: float) -> float:
    return float((Decimal(T) ** 3).sqrt())


def test_pow_1p5_correctly_rounded():
    rng = random.Random(3)
    cases = [rng.uniform(0.05, 50.0) for _ in range(20000)]
    cases += [rng.uniform(1.0, 2.0) * 2.0 ** rng.randint(-300, 300) for _ in range(5000)]
    cases += [4.0, 9.0, 0.25, 1.0, 2.0, 3.0, 0.5]
    for T in cases:
        assert pow_1p5(T) == cr_pow_1p5(T), T


def test_pow_1p5_hard_cases_within_an_ulp():
    """Arguments whose T^1.5 lies within ~2^-104 of a rounding midpoint (T a
    few ulps from 1 or 4: T = 1 + d gives 1 + 1.5 d + 0.375 d^2, a midpoint
    plus a term below the method's resolution) may round the other way:
    never by more than one ulp."""
    for T in (math.nextafter(1.0, 0.0), math.nextafter(1.0, 2.0), math.nextafter(4.0, 5.0),
              1.0 + 3 * 2.0 ** -52, 1.0 - 5 * 2.0 ** -53):
        a, b = pow_1p5(T), cr_pow_1p5(T)
        assert a == b or math.nextafter(a, b) == b, T


def test_host_pow_agrees_with_pow_1p5():
    """On the temperatures of the benchmark flows (non-dimensional T near
    1/(gamma Ma^2 R) ~ 1..10) the host pow is correctly rounded on all but a
    few tenths of a percent of arguments; T * sqrt(T) misses on ~25%."""
    rng = random.Random(5)
    N = 20000
    miss_pow = miss_naive = 0
    for _ in range(N):
        T = rng.uniform(0.5, 12.0)
        ref = pow_1p5(T)
        miss_pow += T ** 1.5 != ref
        miss_naive += T * math.sqrt(T) != ref
    assert miss_pow / N < 0.01, miss_pow / N
    assert miss_naive / N > 0.1
