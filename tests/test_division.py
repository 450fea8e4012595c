"""The Siddon set-up's division (ddiv_r in fir_b200/csrc/siddon.cuh), replayed
on the CPU in exact rational arithmetic: every product, fused multiply-add
and the reciprocal rounded once to the nearest double, as the device's
__dmul_rn, __fma_rn and __drcp_rn do.  The result must be the correctly
rounded quotient a / b (Python's float division is IEEE's) for the operands
the traversal meets: coordinates, plane positions and differences from
1e-6 to 1e4 mm, including divisors close to powers of two and quotients
close to binade boundaries.  For an infinite or NaN operand the device keeps
RN(a RN(1/b)); those cases are checked against IEEE division too.  The GPU
parity tests compare the traversal itself with the oracle."""
import math
from fractions import Fraction

import numpy as np


def fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def ddiv_r(a: float, b: float) -> float:
    """The device sequence: q0 = RN(a rb) with rb = RN(1/b), then two
    corrections by the exact remainder; q0 where the result is NaN."""
    if not (math.isfinite(a) and math.isfinite(b)):
        rb = 1.0 / b if b != 0 else math.copysign(math.inf, b)
        with np.errstate(all="ignore"):
            return float(np.float64(a) * np.float64(rb))
    rb = float(Fraction(1) / Fraction(b))
    q0 = float(Fraction(a) * Fraction(rb))
    q = q0
    for _ in range(2):
        r = fma(-b, q, a)
        q = fma(r, rb, q)
    return q


def same(x: float, y: float) -> bool:
    return (math.isnan(x) and math.isnan(y)) or (x == y and math.copysign(1, x) == math.copysign(1, y))


def test_random_operands_correctly_rounded():
    rng = np.random.default_rng(3)
    n = 20000
    a = rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-6, 4, n)
    b = rng.uniform(-1, 1, n) * 10.0 ** rng.uniform(-5, 4, n)
    bad = [(x, y) for x, y in zip(a.tolist(), b.tolist()) if not same(ddiv_r(x, y), x / y)]
    assert not bad, bad[:5]


def test_hard_divisors_and_quotients():
    rng = np.random.default_rng(4)
    cases = []
    for e in range(-17, 14):
        p = 2.0 ** e
        for b in (p, np.nextafter(p, 0), np.nextafter(p, np.inf), -p, 1.5 * p, 3.0 * p):
            for m in rng.uniform(0.5, 2.0, 12).tolist() + [1.0, np.nextafter(1.0, 2), np.nextafter(1.0, 0)]:
                cases.append((float(m * b * (1 + 2 ** -40)), float(b)))
                cases.append((float(m), float(b)))
    # operands of the kind the set-up forms: plane minus end point over a
    # coordinate difference, and a voxel extent over it
    lo = rng.uniform(-300, 300, 5000)
    c1 = rng.uniform(-500, 500, 5000)
    df = rng.choice([-1, 1], 5000) * 10.0 ** rng.uniform(-5, 3, 5000)
    cases += list(zip((lo - c1).tolist(), df.tolist()))
    cases += [(1.7, float(d)) for d in df[:2000]]
    bad = [(x, y) for x, y in cases if not same(ddiv_r(x, y), x / y)]
    assert not bad, bad[:5]


def test_non_finite_operands_match_ieee():
    vals = [math.inf, -math.inf, math.nan, 0.0, -0.0, 3.5, -2.25, 1e-5]
    for a in vals:
        for b in vals:
            if b == 0.0:
                continue
            with np.errstate(all="ignore"):
                want = float(np.float64(a) / np.float64(b))
            if math.isfinite(a) and math.isfinite(b):
                continue
            assert same(ddiv_r(a, b), want), (a, b)
