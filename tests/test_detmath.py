"""Accuracy of the deterministic functions that the kernels, the host decode
tables and the oracle share (vqm_b200/csrc/ss2_detmath.h), against
double-precision libm, and on samples against exact rational and 40-digit
decimal arithmetic (no libm in the checker: the oracle shares these
functions with the kernels, so they are pinned independently here).

pow, cbrt, exp and sin(pi x) evaluate to ~3e-13 and round once, so they must
land on the correctly rounded float in all but a tiny fraction of cases, and
never more than one ulp away. powf_gamma (the power-law transfers' power)
works in float pairs to ~2^-30: never more than one ulp away, off the
correctly rounded float for well under 1 % of its arguments."""

import ctypes

import numpy as np
import pytest

from oracle import binding as ob


def det(fn, x, y=0.0):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    assert ob.lib().ss2o_detmath(fn, x.ctypes.data_as(ctypes.c_void_p), ctypes.c_float(y),
                                 out.ctypes.data_as(ctypes.c_void_p), x.size) == 0
    return out


def ulps(a, b):
    ai = a.view(np.int32).astype(np.int64)
    bi = b.view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


def check(got, exact64, max_bad_frac=1e-5):
    want = exact64.astype(np.float32)
    d = ulps(got, want)
    assert d.max() <= 1, (d.max(), got[d.argmax()], exact64[d.argmax()])
    assert (d > 0).mean() <= max_bad_frac


def samples(lo, hi, n=2_000_000, seed=0):
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.float32)
    return x


def test_cbrt():
    x = np.concatenate([samples(1e-38, 1e30), samples(0.0037, 1.2),
                        np.float32([1, 8, 27, 0.125, 1e-45, 3e38])])
    check(det(0, x), np.cbrt(x.astype(np.float64)))
    assert det(0, np.float32([0.0, -1.0]))[0] == 0.0


@pytest.mark.parametrize("y", [2.4, 2.2, 2.8, 2.6, 1 / 0.45, 0.2, 1 / 78.84375,
                               1 / 0.1593017578125])
def test_pow(y):
    yf = np.float32(y)
    x = samples(1e-6, 1.5)
    check(det(1, x, yf), np.power(x.astype(np.float64), np.float64(yf)))
    assert det(1, np.float32([0.0, 1.0]), yf).tolist() == [0.0, 1.0]


def test_powf_gamma_exhaustive_for_gamma_2_4():
    """The power-law transfers' single-precision power, on every float of
    its fast range [2^-30, 2^16) for VQM's gamma 2.4: never more than one ulp
    from the correctly rounded power, and on it for all but ~0.35 %."""
    yf = np.float32(2.4)
    lo = int(np.float32(2.0 ** -30).view(np.uint32))
    hi = int(np.float32(65536.0).view(np.uint32))
    off = total = 0
    for start in range(lo, hi, 1 << 23):
        x = np.arange(start, min(start + (1 << 23), hi), dtype=np.uint32).view(np.float32)
        want = np.power(x.astype(np.float64), np.float64(yf)).astype(np.float32)
        d = ulps(det(5, x, yf), want)
        assert d.max() <= 1, (start, d.max())
        off += int((d > 0).sum())
        total += x.size
    assert off / total < 0.005


@pytest.mark.parametrize("y", [2.2, 2.8, 1.0, 4.0, 1 / 0.45, 2.6])
def test_powf_gamma(y):
    yf = np.float32(y)
    x = samples(2.0 ** -30, 65535.9, n=1_000_000)
    d = ulps(det(5, x, yf), np.power(x.astype(np.float64), np.float64(yf)).astype(np.float32))
    assert d.max() <= 1 and (d > 0).mean() < 0.01
    # Below 2^-30 it is 0 for y in [2, 4] (the exact power is below 2^-60);
    # from 2^16 up, and for y outside [2, 4], it is pow itself.
    tiny = np.float32([0.0, 1e-12, 2.0 ** -31, np.nextafter(np.float32(2.0 ** -30), 0)])
    big = np.float32([65536.0, 1e6])
    if 2.0 <= yf <= 4.0:
        assert np.all(det(5, tiny, yf) == 0.0)
        assert det(5, np.float32([2.0 ** -30]), yf)[0] > 0.0
    else:
        assert np.array_equal(det(5, tiny, yf), det(1, tiny, yf))
    assert np.array_equal(det(5, big, yf), det(1, big, yf))
    assert det(5, np.float32([1.0]), yf)[0] == 1.0
    assert np.array_equal(det(5, x[:1000], np.float32(0.5)), det(1, x[:1000], np.float32(0.5)))


def test_divf_matches_ieee_division():
    """The maps' division (seeded reciprocal, three Newton steps, one
    residual correction) over its domain, b in [2^-20, 2^20], |a| < 2^20:
    equal to IEEE single-precision division on every sampled quotient (60
    divisors x 50,000 dividends) and on every dividend of the binade [1, 2)
    for a spread of divisors."""
    rng = np.random.default_rng(7)
    for b in np.exp(rng.uniform(np.log(2.0 ** -20), np.log(2.0 ** 20), 60)).astype(np.float32):
        a = (rng.uniform(-1, 1, 50_000) *
             np.exp(rng.uniform(np.log(1e-7), np.log(2.0 ** 20), 50_000))).astype(np.float32)
        assert np.array_equal(det(6, a, b), a / b)
    a = np.arange(0x3F800000, 0x40000000, dtype=np.uint32).view(np.float32)
    for b in np.float32([1.0, 1.5, 0.0009, 0.3337, 7.25, 2.0 ** -19, 1234.5]):
        assert np.array_equal(det(6, a, b), a / b)
    assert det(6, np.float32([0.0]), np.float32(3.0))[0] == 0.0


def test_pow_base10():
    # 10^(2 (v - 1)) and 10^(2.5 (v - 1)) of the log transfers.
    e = np.random.default_rng(1).uniform(-5, 0, 200_000).astype(np.float32)
    x = np.full_like(e, 10.0)
    out = np.array([det(1, x[i:i + 1], float(e[i]))[0] for i in range(0, 2000)])
    check(out, np.power(10.0, e[:2000].astype(np.float64)), max_bad_frac=1e-3)


def test_exp():
    x = np.random.default_rng(2).uniform(-20, 20, 1_000_000).astype(np.float32)
    check(det(2, x), np.exp(x.astype(np.float64)))


def test_sinpi():
    x = np.random.default_rng(3).uniform(0, 3, 1_000_000).astype(np.float32)
    x = np.concatenate([x, np.float32([0.0, 1.0, 2.0, 1e-7, 2.0000002])])
    got = det(3, x)
    exact = np.sin(np.pi * x.astype(np.float64))
    # sin(pi x) has zeros at integers; compare with an absolute floor there.
    want = exact.astype(np.float32)
    d = ulps(got, want)
    near_zero = np.abs(exact) < 1e-6
    assert d[~near_zero].max() <= 1
    assert np.abs(got[near_zero] - exact[near_zero]).max() < 1e-12


def test_cbrt_every_float_of_three_binades():
    # The seed and every step scale exactly by 2^k when x scales by 2^3k, so
    # [1, 8) covers the unscaled path's behaviour for every float: each one
    # must be the correctly rounded cube root.
    u = np.arange(np.float32(1.0).view(np.uint32), np.float32(8.0).view(np.uint32),
                  dtype=np.uint32)
    x = u.view(np.float32)
    got = det(0, x)
    want = np.cbrt(x.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_round_half_matches_ieee_binary16():
    rng = np.random.default_rng(7)
    x = np.concatenate([
        rng.uniform(-2, 2, 1_000_000), np.exp(rng.uniform(np.log(1e-9), np.log(7e4), 500_000)),
        np.float32([0.0, -0.0, 65504.0, 65519.0, 65520.0, 6.0e-8, 2.98e-8, 6.1035e-5,
                    np.inf, -np.inf])]).astype(np.float32)
    want = x.astype(np.float16).astype(np.float32)
    got = det(4, x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_prepare_cube_root_equals_the_shared_one_on_its_whole_range():
    """The prepare kernels seed x^(-1/3) from the special-function unit and
    take one Newton step where ss2dm::cbrt takes three from a bit-level
    seed; both end in the same exact-residual correction and round once.
    They must give the same float on every input of the band that route
    takes, [2^-16, 2^24) (335 M values), checked on the device; outside it
    they part at one hard-to-round mantissa every third octave."""
    from vqm_b200 import ss2
    lo = int(np.float32(2.0 ** -16).view(np.uint32))
    hi = int(np.float32(2.0 ** 24).view(np.uint32)) - 1
    mismatches, first_bad = ss2.check_cbrt(lo, hi)
    assert mismatches == 0, hex(first_bad)
    # Just outside the band the two routes part at 0x7afd13 (the route is
    # not taken there), which also shows that the check sees differences.
    below = int(np.float32(2.0 ** -17).view(np.uint32))
    assert ss2.check_cbrt(below, lo - 1) == (1, below | 0x7AFD13)



@pytest.mark.gpu
def test_blur_division_equals_the_shared_one_across_its_band():
    """The blur's maps take the divisor's reciprocal from the special-function
    unit and one Newton step, where the shared division takes three from a bit
    seed; both then correct the quotient with its exact residual, which
    absorbs the reciprocals' occasional 1-ulp difference. Checked on the
    device for every divisor of the maps' band [2^-11, 2^4] (126 M values) at
    sixteen quotient values each: 2 G divisions."""
    from vqm_b200 import ss2
    lo = int(np.float32(2.0 ** -11).view(np.uint32))
    hi = int(np.float32(2.0 ** 4).view(np.uint32))
    mismatches, first_bad = ss2.check_division(lo, hi)
    assert mismatches == 0, (mismatches, hex(first_bad))


def test_cbrt_correctly_rounded_by_exact_arithmetic():
    """The cube root's correct rounding checked without libm: for float x
    and the returned float y with ulp u, exact rational arithmetic confirms
    (y - u/2)^3 <= x <= (y + u/2)^3 on 60,000 random floats of [1, 8) and of
    the whole normal range."""
    from fractions import Fraction
    rng = np.random.default_rng(31)
    lo, hi = np.float32(1.0).view(np.uint32), np.float32(8.0).view(np.uint32)
    x = np.concatenate([
        rng.integers(lo, hi, 30_000, dtype=np.uint32).view(np.float32),
        samples(1.2e-38, 3e38, n=30_000, seed=32)])
    y = det(0, x)
    for xi, yi in zip(x.tolist(), y.tolist()):
        m, e = np.frexp(np.float32(yi))  # yi = m 2^e, m in [0.5, 1)
        half_ulp = Fraction(2) ** (int(e) - 25)
        fy, fx = Fraction(yi), Fraction(xi)
        assert (fy - half_ulp) ** 3 <= fx <= (fy + half_ulp) ** 3, (xi, yi)


def test_powers_faithful_by_decimal_arithmetic():
    """pow and the transfers' powf_gamma checked without libm: each result
    is one of the two floats around the exact power, computed in 40-digit
    decimal arithmetic, on 4,000 random arguments per exponent."""
    import decimal
    ctx = decimal.Context(prec=40)
    for fn, y, lo, hi in ((5, 2.4, 2.0 ** -30, 65535.9), (5, 2.2, 1e-6, 1.5),
                          (1, 1 / 0.45, 1e-6, 1.5), (1, 1 / 78.84375, 1e-6, 1.0),
                          (1, 1 / 0.1593017578125, 1e-3, 1.0)):
        yf = np.float32(y)
        x = samples(lo, hi, n=4_000, seed=int(1e3 * y))
        got = det(fn, x, yf)
        for xi, gi in zip(x.tolist(), got.tolist()):
            exact = ctx.power(decimal.Decimal(xi), decimal.Decimal(float(yf)))
            below = np.float32(float(exact))
            if decimal.Decimal(float(below)) > exact:
                below = np.nextafter(below, np.float32(0))
            above = np.nextafter(below, np.float32(np.inf))
            assert gi in (float(below), float(above)), (fn, y, xi, gi, exact)
