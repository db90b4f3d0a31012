"""The step's division by a shared divisor (div_rn in harm_phys.cuh): a restatement
of its steps in exact rational arithmetic on the CPU, against Python's IEEE double
division, and (GPU) the device routine itself against the device's IEEE division.

div_rn(a, b, y), y = RN(1/b): q = RN(a y); r = RN(a - b q) (one FMA);
q = RN(q + r y) (one FMA); r = a - b q (exact); q moves one step towards a/b
when |r| exceeds b times half the gap between q and that neighbour."""
import math
import random
import struct
from fractions import Fraction

import pytest


def bits(x):
    return struct.unpack("<q", struct.pack("<d", x))[0]


def from_bits(i):
    return struct.unpack("<d", struct.pack("<q", i))[0]


def fma(a, b, c):
    """a*b + c rounded once to the nearest double (float() of a Fraction rounds
    to nearest, ties to even)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def div_rn(a, b, y):
    ia = bits(a)
    ea = (ia >> 52) & 0x7FF
    eb = (bits(b) >> 52) & 0xFFF
    okb = 963 <= eb <= 1083
    if not okb or not (223 <= ea <= 1823):
        if okb and (ia & 0x7FFFFFFFFFFFFFFF) == 0:
            return a * y
        return a / b
    q = a * y
    r = fma(-q, b, a)
    q = fma(r, y, q)
    return finish(a, b, q)


def finish(a, b, q):
    """The last step: q is one of the two doubles around a/b (faithful)."""
    r = fma(-q, b, a)
    iq = bits(q)
    up = (r > 0.) == (q > 0.)
    eq = (iq >> 52) & 0x7FF
    eh = eq - 53 - (1 if (not up and (iq & 0xFFFFFFFFFFFFF) == 0) else 0)
    hb = from_bits(eh << 52) * b
    if abs(r) > hb:
        q = from_bits(iq + (1 if up else -1))
    return q


def rand_double(rng, emin, emax, neg=None):
    m = rng.getrandbits(52)
    e = rng.randint(emin, emax)
    s = rng.getrandbits(1) if neg is None else int(neg)
    return from_bits((s << 63) | ((e + 1023) << 52) | m) if not s else -from_bits(((e + 1023) << 52) | m)


def test_div_rn_restatement_matches_ieee_division():
    rng = random.Random(20240611)
    n_mid = 0
    for t in range(60000):
        eb = rng.randint(-60, 60)
        if t % 5 == 0:
            b = from_bits(((eb + 1023) << 52) | 0xFFFFFFFFFFFFF)
        else:
            b = rand_double(rng, eb, eb, neg=False)
        y = 1. / b
        if t % 2 == 0:
            a = rand_double(rng, -820, 820)
        else:
            # a/b within a tiny distance of the midpoint q + ulp(q)/2
            q = rand_double(rng, -60, 60)
            hulp = from_bits((((bits(q) >> 52) & 0x7FF) - 53) << 52)
            a = float(Fraction(b) * (Fraction(q) + Fraction(hulp) * rng.choice((1, -1))))
            n_mid += 1
        got, want = div_rn(a, b, y), a / b
        assert bits(got) == bits(want), (a, b, got, want)
    assert n_mid == 30000


def test_last_step_picks_the_nearest_of_two_faithful_quotients():
    """The correction that decides the last bit, fed both neighbours of a/b,
    including quotients just above and below powers of two (where the gap
    below is half the gap above)."""
    rng = random.Random(77)
    for t in range(40000):
        b = rand_double(rng, -60, 60, neg=False)
        if t % 4 == 0:
            # a/b within a few ulps of a power of two
            z0 = Fraction(2) ** rng.randint(-50, 50) * rng.choice((1, -1))
            a = float(Fraction(b) * z0 * (1 + Fraction(rng.randint(-8, 8), 2 ** 53)))
        else:
            a = rand_double(rng, -700, 700)
        want = a / b
        z = Fraction(a) / Fraction(b)
        lo = want if Fraction(want) <= z else from_bits(bits(want) - 1 if want > 0 else bits(want) + 1)
        hi = want if Fraction(want) >= z else from_bits(bits(want) + 1 if want > 0 else bits(want) - 1)
        for q in (lo, hi):
            assert bits(finish(a, b, q)) == bits(want), (a, b, q, want)


def test_div_rn_special_numerators():
    b = 0.7
    y = 1. / b
    for a in (0., -0., 5e-324, -5e-324, 1e-250, 1e300, -1e300, math.inf, -math.inf):
        assert bits(div_rn(a, b, y)) == bits(a / b), a
    assert math.isnan(div_rn(math.nan, b, y))
    # divisors outside the fast range divide directly
    for b in (1e-30, 1e30, -0.5):
        assert bits(div_rn(3.0, b, 1. / b)) == bits(3.0 / b)


@pytest.mark.gpu
def test_div_rn_on_device_matches_ieee_division(harm_lib):
    import harm_cool_b200 as hc
    bad, mid = hc.div_check(1 << 31, seed=7)
    assert mid > (1 << 31) // 3
    assert bad == 0
