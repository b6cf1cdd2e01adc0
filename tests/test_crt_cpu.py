"""The residue (Chinese remainder) form of the int8 tensor-core products, on
the CPU: the constants libgwb uses (moduli, inverses, double-double 1/m and
M, the integer bit budget), an exact-integer model of the whole product, and
a bit-level emulation of the device's drain reduction and double-double
reconstruction (every fma evaluated exactly and rounded once)."""

from __future__ import annotations

import math
from fractions import Fraction

import numpy as np
import pytest

from gradwave_b200 import _lib


def _constants(n: int):
    m = np.zeros(n, dtype=np.uint32)
    y = np.zeros(n, dtype=np.uint32)
    ih = np.zeros(n, dtype=np.float64)
    il = np.zeros(n, dtype=np.float64)
    mhl = np.zeros(2, dtype=np.float64)
    _lib.call("gwb_crt_constants", n, m.ctypes.data, y.ctypes.data, ih.ctypes.data, il.ctypes.data,
              mhl.ctypes.data)
    return [int(v) for v in m], [int(v) for v in y], ih, il, mhl, int(_lib.load().gwb_crt_bits(n))


def _fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _two_sum(a: float, b: float):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def _reconstruct(r: list[int], ih, il, mh: float, ml: float) -> float:
    """k_crt_reduce on one element: r[t] = (C y_t) mod m_t summed over splits."""
    sh = sl = 0.0
    for t, R in enumerate(r):
        rr = float(R)
        ph = rr * float(ih[t])
        pl = _fma(rr, float(il[t]), _fma(rr, float(ih[t]), -ph))
        sh, e = _two_sum(sh, ph)
        sl += e + pl
    sh -= math.floor(sh)
    f, fl = _two_sum(sh, sl)
    if f >= 0.5:
        f -= 1.0
    if f < -0.5:
        f += 1.0
    return _fma(f, mh, _fma(f, ml, fl * mh))


def _mod_u32(u: int, m: int, mg: int) -> int:
    q = (u * mg) >> 39
    r = u - q * m
    return r + m if r < 0 else r


@pytest.mark.parametrize("n", [16, 18, 20])
def test_crt_constants(n):
    mods, y, ih, il, mhl, p = _constants(n)
    assert all(2 <= m <= 256 for m in mods)
    for i in range(n):
        for j in range(i + 1, n):
            assert math.gcd(mods[i], mods[j]) == 1
    M = math.prod(mods)
    for t, m in enumerate(mods):
        assert (M // m * y[t]) % m == 1
        assert abs(Fraction(float(ih[t])) + Fraction(float(il[t])) - Fraction(1, m)) < Fraction(1, m) * 2.0 ** -104
    assert abs(Fraction(float(mhl[0])) + Fraction(float(mhl[1])) - M) < M * 2.0 ** -100
    # |C| < 2^19 2^2p must stay below M / 2
    assert 2 * p + 19 <= math.log2(M) - 1
    assert p == {16: 52, 18: 60, 20: 67}[n]
    assert _lib.load().gwb_crt_bits(17) == -1


def test_crt_model_product_is_exact():
    """Exact-integer model: centred residues of |x| < 2^p, one product per
    modulus reduced and times y_t, then frac(sum r_t / m_t) M = A B^T."""
    n = 18
    mods, y, ih, il, mhl, p = _constants(n)
    M = math.prod(mods)
    rng = np.random.default_rng(5)
    K = 40
    lim = 2 ** p
    a = [[int(v) for v in row] for row in rng.integers(-lim + 1, lim, size=(3, K), dtype=np.int64)]
    b = [[int(v) for v in row] for row in rng.integers(-lim + 1, lim, size=(4, K), dtype=np.int64)]
    a[0] = [lim - 1] * K          # extreme rows: the largest magnitudes, both signs
    b[0] = [-(lim - 1)] * K

    def centred(x, m):
        r = x % m
        return r - m if r > (m - 1) // 2 else r

    for i in range(3):
        for j in range(4):
            exact = sum(a[i][k] * b[j][k] for k in range(K))
            rs = []
            for t, m in enumerate(mods):
                ct = sum(centred(a[i][k], m) * centred(b[j][k], m) for k in range(K))
                assert abs(ct) < 2 ** 31
                rs.append((ct % m) * y[t] % m)
            frac = sum(Fraction(r, m) for r, m in zip(rs, mods)) % 1
            if frac >= Fraction(1, 2):
                frac -= 1
            assert frac * M == exact
            # the device's double-double evaluation of the same sum
            got = _reconstruct(rs, ih, il, float(mhl[0]), float(mhl[1]))
            assert abs(Fraction(got) - exact) <= abs(exact) * 2.0 ** -52 + 2.0 ** 44


def test_crt_drain_reduction():
    """The drain's modular arithmetic on int32 accumulators: (x + 2^31) mod m
    by the 2^39 multiplier, minus 2^31 mod m, times y_t, mod m."""
    mods, y, *_ = _constants(20)
    rng = np.random.default_rng(1)
    xs = [-2 ** 31, -2 ** 31 + 1, -1, 0, 1, 2 ** 31 - 1] + [int(v) for v in rng.integers(-2 ** 31, 2 ** 31, 2000)]
    for t, m in enumerate(mods):
        mg = (1 << 39) // m + 1
        assert mg < 2 ** 32
        c31 = (1 << 31) % m
        for x in xs:
            u = (x + 2 ** 31) & 0xFFFFFFFF
            v = _mod_u32(u, m, mg) + m - c31
            assert v * y[t] < 2 ** 32
            w = _mod_u32(v * y[t], m, mg)
            assert 0 <= w < m
            assert w == (x * y[t]) % m


def test_crt_split_residue_rule():
    """The split kernels' residue of an integer-valued double: q = rint(x / m)
    (rounded product with the rounded 1/m), x - q m by one fma, then centred."""
    for n, bits in ((16, 52), (18, 60), (20, 67)):
        mods, *_ = _constants(n)
        rng = np.random.default_rng(n)
        vals = [0.0, 1.0, -1.0, float(2 ** bits - 2 ** (bits - 52)), -float(2 ** bits - 2 ** (bits - 52))]
        vals += [float(np.ldexp(np.rint(v * 2.0 ** 52), bits - 52)) for v in rng.uniform(-1, 1, 200)]
        for x in vals:
            for m in mods:
                q = float(np.rint(x * (1.0 / m)))
                r = _fma(-q, float(m), x)
                assert r == int(r) and abs(r) < 2 ** 15
                ri = int(math.fmod(int(r), m))
                if ri > (m - 1) // 2:
                    ri -= m
                elif ri < -(m // 2):
                    ri += m
                assert -128 <= ri <= 127
                assert (ri - int(x)) % m == 0
