"""Integer model of the double-precision Montgomery products (csrc/field_f64.cuh: mont_mul,
mont_mul_sub), run on the CPU to pin the bounds the accumulation kernel relies on.

The model follows the device code step by step. A limb product a*b (< 2^104) splits into the bit
patterns 0x467.. + floor(ab / 2^52) (the high-half FMA, rounded toward zero) and 0x433.. +
(ab mod 2^52) (the low-half FMA, exact); column sums are 64-bit integers that wrap (unsigned for
mont_mul, signed for mont_mul_sub), so the model wraps them the same way. What it checks: the
result is congruent to the product times 2^-260 modulo the field prime, and stays below the
bound stated in the source (2p for mont_mul, 1.3p for mont_mul_sub with a, b < 4p, c, d < 2p)."""
import random

from oracle.bn254 import Q as P, R as R_PRIME

B52, B104 = 0x4330000000000000, 0x4670000000000000
M52, M64 = (1 << 52) - 1, (1 << 64) - 1
R260 = 1 << 260


def limbs(x):
    return [(x >> (52 * i)) & M52 if i < 4 else x >> 208 for i in range(5)]


def value(l):
    return sum(v << (52 * i) for i, v in enumerate(l))


def split(a, b):
    """Bit patterns of the high-half and low-half FMAs of one limb product."""
    ab = a * b
    assert ab < 1 << 104
    return B104 + (ab >> 52), B52 + (ab & M52)


def wrap_u(v):
    return v & M64


def wrap_s(v):
    v &= M64
    return v - (1 << 64) if v >> 63 else v


def reduce_columns(col, mod, wrap):
    """The reduction phase and the final carry pass, shared by both products."""
    pl = limbs(mod)
    pinv = (-pow(mod, -1, 1 << 52)) % (1 << 52)
    for i in range(5):
        t = col[i]
        carry = (t + M52) >> 52  # ceil(t / 2^52) (arithmetic shift when signed)
        q = ((t & M52) * pinv) & M52
        h0, _ = split(q, pl[0])
        col[i + 1] = wrap(col[i + 1] + h0 + carry)
        for j in range(1, 5):
            h, lo = split(q, pl[j])
            col[i + j] = wrap(col[i + j] + lo)
            col[i + j + 1] = wrap(col[i + j + 1] + h)
    out, carry = [], 0
    for k in range(5, 10):
        v = col[k] + carry
        carry = v >> 52
        out.append(v & M52 if k < 9 else v)
    return value(out)


def lo_terms(k):
    return sum(1 for i in range(5) for j in range(5) if i + j == k) + \
        sum(1 for i in range(5) for j in range(1, 5) if i + j == k)


def hi_terms(k):
    return 2 * sum(1 for i in range(5) for j in range(5) if i + j + 1 == k)


def red_bias(k):
    lo = sum(1 for i in range(5) for j in range(1, 5) if i + j == k)
    hi = sum(1 for i in range(5) for j in range(5) if i + j + 1 == k)
    return lo * B52 + hi * B104


def mont_mul(x, y, mod):
    a, b = limbs(x), limbs(y)
    col = [wrap_u(-(lo_terms(k) * B52 + hi_terms(k) * B104)) for k in range(10)]
    for i in range(5):
        for j in range(5):
            h, lo = split(a[i], b[j])
            col[i + j] = wrap_u(col[i + j] + lo)
            col[i + j + 1] = wrap_u(col[i + j + 1] + h)
    return reduce_columns(col, mod, wrap_u)


def mont_mul_sub(x, y, z, w, mod):
    a, b, c, d = limbs(x), limbs(y), limbs(z), limbs(w)
    m = [((mod << 256) >> (52 * k)) & M52 if k < 9 else (mod << 256) >> 468 for k in range(10)]
    col = [wrap_s(m[k] - red_bias(k)) for k in range(10)]
    for i in range(5):
        for j in range(5):
            h, lo = split(a[i], b[j])
            h2, l2 = split(c[i], d[j])
            col[i + j] = wrap_s(col[i + j] + lo - l2)
            col[i + j + 1] = wrap_s(col[i + j + 1] + h - h2)
    return reduce_columns(col, mod, wrap_s)


def check_mul(x, y, mod):
    r = mont_mul(x, y, mod)
    assert (r - x * y * pow(R260, -1, mod)) % mod == 0
    assert r < 2 * mod
    return r


def test_mont_mul_congruent_and_below_2p():
    rng = random.Random(1)
    for mod in (P, R_PRIME):
        edge = [0, 1, mod - 1, mod, 2 * mod - 1, (1 << 256) - 1, (1 << 255) + 12345]
        for x in edge:
            for y in edge:
                check_mul(x, y, mod)
        for _ in range(3000):
            check_mul(rng.getrandbits(256), rng.getrandbits(256), mod)


def test_mont_mul_sub_congruent_and_below_1_3p():
    rng = random.Random(2)
    worst = 0
    cases = [(4 * P - 1, 4 * P - 1, 0, 0), (0, 0, 2 * P - 1, 2 * P - 1), (4 * P - 1, 4 * P - 1, 2 * P - 1, 2 * P - 1),
             (0, 0, 0, 0), (1, 1, 1, 1)]
    cases += [(rng.randrange(4 * P), rng.randrange(4 * P), rng.randrange(2 * P), rng.randrange(2 * P))
              for _ in range(3000)]
    for x, y, z, w in cases:
        r = mont_mul_sub(x, y, z, w, P)
        assert (r - (x * y - z * w) * pow(R260, -1, P)) % P == 0
        assert r < 13 * P // 10
        worst = max(worst, r)
    assert worst > P  # the bound is not vacuous: results above p do occur


def test_shifted_modulus_columns():
    """p 2^256 in base-2^52 columns equals the limbs of p << 48 placed from column 4 (the
    compile-time table of the device code)."""
    for mod in (P, R_PRIME):
        m = [((mod << 256) >> (52 * k)) & M52 if k < 9 else (mod << 256) >> 468 for k in range(10)]
        pl = limbs(mod)
        table = [0] * 4 + [((pl[j - 1] >> 4) if j >= 1 else 0) | (((pl[j] & 0xF) << 48) if j < 5 else 0)
                           for j in range(6)]
        assert m == table
