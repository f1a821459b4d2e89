"""The kernels divide by rscale and by 3 with a known-divisor division (a
double-word reciprocal quotient plus one remainder correction) instead of the
general IEEE division the reference's numpy code performs
(kernels/horizontalizevec.py:51-54, kernels/oprtdiffusion.py:59-134).  The
result must carry the same bits as x / b.

The CPU test restates the method with exact rational arithmetic for the fused
multiply-adds and checks it on random and near-midpoint quotients (the cases
where a faithful but not correctly rounded quotient would show); the GPU test
runs the device routine (nc_divide_known) on ten million values per divisor,
and on per-element divisors with the reciprocal formed on the device."""
from __future__ import annotations

import math
import random
from fractions import Fraction

import numpy as np
import pytest

RSCALE = 6371220.0   # the earth radius of every workload


def _fma(a: float, b: float, c: float) -> float:
    r = Fraction(a) * Fraction(b) + Fraction(c)
    if r != 0:
        return float(r)   # Fraction -> float rounds to nearest, ties to even
    neg = (math.copysign(1.0, a) * math.copysign(1.0, b) < 0) and math.copysign(1.0, c) < 0
    return -0.0 if neg else 0.0


def _recip_pair(b: float):
    h = 1.0 / b
    return h, float(Fraction(1) / Fraction(b) - Fraction(h))


def _recip_runtime(b: float):
    """the device form for a divisor known only at run time: RN(1/b) and the
    tail RN((1 - b*RN(1/b)) * RN(1/b))"""
    h = 1.0 / b
    return h, _fma(-h, b, 1.0) * h


def _div_by(x: float, b: float, bh: float, bl: float) -> float:
    q0 = _fma(x, bh, x * bl)
    r = _fma(-q0, b, x)
    q = _fma(r, bh, q0)
    return x * bh if x == 0.0 else q


def _cases(b: float, n: int, rng: random.Random):
    for t in range(n):
        if t % 2 == 0:
            yield rng.uniform(-1.0, 1.0) * 2.0 ** rng.randint(-60, 60)
        else:   # quotient next to a midpoint between two doubles
            m = rng.uniform(1.0, 2.0) * 2.0 ** rng.randint(-40, 40)
            x0 = float((Fraction(m) + Fraction(math.ulp(m)) / 2) * Fraction(b))
            yield x0 + rng.choice((-1, 0, 1)) * math.ulp(x0)


def _bits(v: float) -> int:
    return int(np.float64(v).view(np.uint64))


@pytest.mark.parametrize("b", [3.0, RSCALE, -3.0, 637122.0, 1.0e-3])
def test_method_matches_ieee_division(b):
    rng = random.Random(17)
    bh, bl = _recip_pair(b)
    bad = [x for x in _cases(b, 6000, rng) if _bits(_div_by(x, b, bh, bl)) != _bits(x / b)]
    assert not bad, bad[:5]


def test_method_random_divisors():
    rng = random.Random(5)
    for _ in range(30):
        b = rng.uniform(1.0, 2.0) * 2.0 ** rng.randint(-30, 30)
        bh, bl = _recip_pair(b)
        for x in _cases(b, 400, rng):
            assert _bits(_div_by(x, b, bh, bl)) == _bits(x / b), (x, b)


def test_method_runtime_reciprocal():
    rng = random.Random(9)
    for _ in range(60):
        b = rng.uniform(1.0, 2.0) * 2.0 ** rng.randint(-40, 40)
        bh, bl = _recip_runtime(b)
        for x in _cases(b, 300, rng):
            assert _bits(_div_by(x, b, bh, bl)) == _bits(x / b), (x, b)


def test_method_signed_zero():
    for b in (3.0, -3.0, RSCALE):
        for bh, bl in (_recip_pair(b), _recip_runtime(b)):
            for x in (0.0, -0.0):
                assert _bits(_div_by(x, b, bh, bl)) == _bits(x / b)


def _device_cases(b: float, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    wide = rng.uniform(-1.0, 1.0, n) * np.exp2(rng.integers(-200, 200, n)).astype(np.float64)
    m = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-60, 60, n)).astype(np.float64)
    half = (np.nextafter(m, np.inf) - m) / 2
    near = ((m.astype(np.longdouble) + half.astype(np.longdouble)) * np.longdouble(b)).astype(np.float64)
    near = np.concatenate([np.nextafter(near, -np.inf), near, np.nextafter(near, np.inf)])
    ints = rng.integers(-(2 ** 53), 2 ** 53, n).astype(np.float64)
    return np.concatenate([wide, near, ints, [0.0, -0.0, 1.0, -1.0, 3.0, RSCALE]])


@pytest.mark.gpu
@pytest.mark.parametrize("b", [3.0, RSCALE, -7.25e-4])
def test_device_division_matches_ieee(pkg, b):
    x = _device_cases(b, 2_000_000, 3)
    q = pkg.runtime.divide_known(x, b)
    want = x / b
    diff = np.flatnonzero(q.view(np.uint64) != want.view(np.uint64))
    assert diff.size == 0, (x[diff[:5]], q[diff[:5]], want[diff[:5]])


@pytest.mark.gpu
def test_device_division_per_element_divisors(pkg):
    rng = np.random.default_rng(11)
    n = 2_000_000
    y = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-30, 30, n)).astype(np.float64)
    x = rng.uniform(-1.0, 1.0, n) * np.exp2(rng.integers(-200, 200, n)).astype(np.float64)
    m = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-60, 60, n)).astype(np.float64)
    half = (np.nextafter(m, np.inf) - m) / 2
    near = ((m.astype(np.longdouble) + half.astype(np.longdouble)) * y.astype(np.longdouble)).astype(np.float64)
    xs = np.concatenate([x, near, np.nextafter(near, np.inf), [0.0, -0.0]])
    ys = np.concatenate([y, y, y, [3.0, 3.0]])
    q = pkg.runtime.divide_known(xs, ys)
    want = xs / ys
    diff = np.flatnonzero(q.view(np.uint64) != want.view(np.uint64))
    assert diff.size == 0, (xs[diff[:5]], ys[diff[:5]], q[diff[:5]], want[diff[:5]])
