"""BN254 big-integer oracle (pure Python) for the MSM and NTT hot path.

TEST INFRASTRUCTURE ONLY. This module is a checker: only tests, the smoke check and
the CPU-baseline leg of bench.py may import it. Nothing in the product library calls it.

It restates, with Python integers, the mathematics of the reference's path:

* field moduli FQ / FR ............................ src/field.rs:18-20
* modular add/sub/mul/pow/inverse ................. src/host.rs:27-60,100-102
* root of unity 5^((r-1) >> log_n) ................ src/host.rs:94-98
* word packing (8 little-endian u32 per element) .. src/host.rs:104-110
* XYZZ group law (dbl-2008-s-1, madd-2008-s,
  add-2008-s) with every special case ............. src/shaders/curve.wgsl:23-75
* Fq2 = Fq[u]/(u^2+1), mul/sqr .................... src/group.rs:38-48, src/msm.rs:375-387
* signed c-bit digits with carry .................. src/shaders/msm_digits.wgsl:19-37
* Pippenger bucket sums and Horner combine ........ src/shaders/msm_reduce_chunks.wgsl,
                                                     src/shaders/msm_combine.wgsl
* DIF NTT, natural order in/out, inverse with 1/n . src/ntt.rs:26-68, src/shaders/ntt.wgsl:50-73
* xyzz_to_affine / xyzz_to_affine_g2 .............. src/msm.rs:345-387
* GLV split of a G1 scalar (the B200 build's G1 GLV mode; the reference names GLV as its next
  step, README.md:223-224, and has no code for it) ... Gallant, Lambert, Vanstone, CRYPTO
  2001: constants derived below from Q and R alone

Pinned against the reference's golden vectors (tests/golden/{ntt,msm}.json, produced by
ffjavascript 0.3.1, an implementation independent of arkworks) by tests/test_oracle.py.
MSM and NTT outputs are unique mathematical values, so any correct restatement is
bit-identical to arkworks' VariableBaseMSM and Radix2EvaluationDomain::fft.

The BN254 G2 generator below is the standard public one (the same point as arkworks'
`G2Affine::generator()` and EIP-197); the reference only names it through arkworks
(tests/g2.rs:136), so its membership (on the twist, order r) is checked by
`self_check()` instead of against a fixture.
"""
from __future__ import annotations

Q = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47
R = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001
MONT = 1 << 256  # Montgomery radix of the B200 build (the reference's WGSL uses 2^260)

G1_GEN = (1, 2)
G2_GEN = (
    (0x1800DEEF121F1E76426A00665E5C4479674322D4F75EDADD46DEBD5CD992F6ED,
     0x198E9393920D483A7260BFB731FB5D25F1AA493335A9E71297E485B7AEF312C2),
    (0x12C85EA5DB8C6DEB4AAB71808DCB408FE3D1E7690C43D37B4CE6CC0166FA7DAA,
     0x090689D0585FF075EC9E99AD690C3395BC4B313370B38EF355ACDADCD122975B),
)
G1_B = 3


# ---------------------------------------------------------------- words

def words32(x: int) -> list[int]:
    """Integer < 2^256 -> 8 little-endian u32 words (src/host.rs:104-106)."""
    return [(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)]


def from_words32(w) -> int:
    """8 little-endian u32 words -> integer (src/host.rs:108-110)."""
    return sum(int(w[i]) << (32 * i) for i in range(8))


def hex_words(h: str) -> list[int]:
    """Big-endian hex string (golden-vector format) -> 8 LE u32 words
    (tests/golden_vectors/mod.rs:35-40)."""
    return words32(int(h, 16))


# ---------------------------------------------------------------- fields

def inv(x: int, m: int) -> int:
    return pow(x, m - 2, m)


def root_of_unity(log_n: int) -> int:
    """Primitive 2^log_n-th root of unity of Fr with generator 5 (src/host.rs:94-98)."""
    return pow(5, (R - 1) >> log_n, R)


class Fq2:
    """a + b*u with u^2 = -1 over Fq (src/group.rs:38-48)."""
    __slots__ = ("a", "b")

    def __init__(self, a: int, b: int = 0):
        self.a, self.b = a % Q, b % Q

    def __add__(s, o): return Fq2(s.a + o.a, s.b + o.b)
    def __sub__(s, o): return Fq2(s.a - o.a, s.b - o.b)
    def __neg__(s): return Fq2(-s.a, -s.b)
    def __mul__(s, o):
        if isinstance(o, int):
            return Fq2(s.a * o, s.b * o)
        return Fq2(s.a * o.a - s.b * o.b, s.a * o.b + s.b * o.a)
    __rmul__ = __mul__
    def __eq__(s, o): return isinstance(o, Fq2) and s.a == o.a and s.b == o.b
    def __hash__(s): return hash((s.a, s.b))
    def is_zero(s): return s.a == 0 and s.b == 0
    def inv(s):
        """1/(a+bu) = (a-bu)/(a^2+b^2) (src/msm.rs:382-387)."""
        n = inv((s.a * s.a + s.b * s.b) % Q, Q)
        return Fq2(s.a * n, -s.b * n)
    def __repr__(s): return f"Fq2({s.a:#x}, {s.b:#x})"


# Field adapters: the group law below is written once over an abstract field.
class _FqOps:
    zero, one = 0, 1
    @staticmethod
    def add(a, b): return (a + b) % Q
    @staticmethod
    def sub(a, b): return (a - b) % Q
    @staticmethod
    def mul(a, b): return a * b % Q
    @staticmethod
    def is_zero(a): return a == 0
    @staticmethod
    def inv(a): return inv(a, Q)


class _Fq2Ops:
    zero, one = Fq2(0), Fq2(1)
    @staticmethod
    def add(a, b): return a + b
    @staticmethod
    def sub(a, b): return a - b
    @staticmethod
    def mul(a, b): return a * b
    @staticmethod
    def is_zero(a): return a.is_zero()
    @staticmethod
    def inv(a): return a.inv()


FIELD = {"G1": _FqOps, "G2": _Fq2Ops}
G2_B = Fq2(3) * Fq2(9, 1).inv()   # twist constant b' = 3 / (9 + u)


# ---------------------------------------------------------------- XYZZ group law
# Affine points are (x, y) or None (infinity; (0, 0) in memory). XYZZ is (X, Y, ZZ, ZZZ)
# with x = X/ZZ, y = Y/ZZZ; infinity is ZZ = 0 (src/shaders/curve.wgsl:1-20).

def xyzz_inf(F):
    return (F.zero, F.zero, F.zero, F.zero)


def xyzz_from_affine(F, p):
    if p is None:
        return xyzz_inf(F)
    return (p[0], p[1], F.one, F.one)


def xyzz_double(F, p):
    """dbl-2008-s-1 with a = 0 (src/shaders/curve.wgsl:22-33)."""
    x, y, zz, zzz = p
    u = F.add(y, y)
    v = F.mul(u, u)
    w = F.mul(u, v)
    s = F.mul(x, v)
    x2 = F.mul(x, x)
    m = F.add(F.add(x2, x2), x2)
    x3 = F.sub(F.mul(m, m), F.add(s, s))
    y3 = F.sub(F.mul(m, F.sub(s, x3)), F.mul(w, y))
    return (x3, y3, F.mul(v, zz), F.mul(w, zzz))


def xyzz_add_affine(F, p, q):
    """madd-2008-s with all special cases (src/shaders/curve.wgsl:35-53)."""
    if q is None:
        return p
    if F.is_zero(p[2]):
        return xyzz_from_affine(F, q)
    x1, y1, zz1, zzz1 = p
    u2 = F.mul(q[0], zz1)
    s2 = F.mul(q[1], zzz1)
    pp = F.sub(u2, x1)
    r = F.sub(s2, y1)
    if F.is_zero(pp):
        return xyzz_double(F, p) if F.is_zero(r) else xyzz_inf(F)
    ppsq = F.mul(pp, pp)
    ppp = F.mul(pp, ppsq)
    q_ = F.mul(x1, ppsq)
    x3 = F.sub(F.sub(F.mul(r, r), ppp), F.add(q_, q_))
    y3 = F.sub(F.mul(r, F.sub(q_, x3)), F.mul(y1, ppp))
    return (x3, y3, F.mul(zz1, ppsq), F.mul(zzz1, ppp))


def xyzz_add(F, p, q):
    """add-2008-s (src/shaders/curve.wgsl:55-75)."""
    if F.is_zero(q[2]):
        return p
    if F.is_zero(p[2]):
        return q
    u1 = F.mul(p[0], q[2])
    u2 = F.mul(q[0], p[2])
    s1 = F.mul(p[1], q[3])
    s2 = F.mul(q[1], p[3])
    pp = F.sub(u2, u1)
    r = F.sub(s2, s1)
    if F.is_zero(pp):
        return xyzz_double(F, p) if F.is_zero(r) else xyzz_inf(F)
    ppsq = F.mul(pp, pp)
    ppp = F.mul(pp, ppsq)
    q_ = F.mul(u1, ppsq)
    x3 = F.sub(F.sub(F.mul(r, r), ppp), F.add(q_, q_))
    y3 = F.sub(F.mul(r, F.sub(q_, x3)), F.mul(s1, ppp))
    return (x3, y3, F.mul(F.mul(p[2], q[2]), ppsq), F.mul(F.mul(p[3], q[3]), ppp))


def xyzz_to_affine_point(F, p):
    if F.is_zero(p[2]):
        return None
    return (F.mul(p[0], F.inv(p[2])), F.mul(p[1], F.inv(p[3])))


def affine_neg(F, p):
    return None if p is None else (p[0], F.sub(F.zero, p[1]))


def affine_add(F, p, q):
    return xyzz_to_affine_point(F, xyzz_add_affine(F, xyzz_from_affine(F, p), q))


def scalar_mul(F, p, k: int):
    """k * P by double-and-add over XYZZ (k reduced mod r first)."""
    k %= R
    acc = xyzz_inf(F)
    for bit in range(k.bit_length() - 1, -1, -1):
        if not F.is_zero(acc[2]):
            acc = xyzz_double(F, acc)
        if (k >> bit) & 1:
            acc = xyzz_add_affine(F, acc, p)
    return xyzz_to_affine_point(F, acc)


def on_curve(group: str, p) -> bool:
    if p is None:
        return True
    F = FIELD[group]
    x, y = p
    b = G1_B if group == "G1" else G2_B
    lhs = F.mul(y, y)
    rhs = F.add(F.mul(F.mul(x, x), x), b)
    return lhs == rhs


# ---------------------------------------------------------------- MSM

def default_window(n: int) -> int:
    """clamp(log2(max(n,1)) - 5, 11, 16) (src/msm.rs:78-80)."""
    return min(max(max(n, 1).bit_length() - 1 - 5, 11), 16)


def signed_digits(s: int, c: int) -> list[int]:
    """Signed c-bit digits of s, W = ceil(255/c) of them, digit in (-2^(c-1), 2^(c-1)]
    (src/shaders/msm_digits.wgsl:19-37): v = window + carry; v >= 2^(c-1) gives v - 2^c
    with a carry into the next window."""
    windows = -(-255 // c)
    half = 1 << (c - 1)
    carry, out = 0, []
    for w in range(windows):
        v = ((s >> (w * c)) & ((1 << c) - 1)) + carry
        carry = 0
        if v >= half:
            v -= 1 << c
            carry = 1
        out.append(v)
    return out


def msm_pippenger(group: str, bases, scalars, c: int | None = None):
    """Signed-digit Pippenger: per window, buckets of |digit|, running-sum reduction
    sum_b (b+1)*bucket_b, then Horner over windows (src/shaders/msm_*.wgsl)."""
    F = FIELD[group]
    n = len(scalars)
    c = c or default_window(n)
    windows = -(-255 // c)
    half = 1 << (c - 1)
    digits = [signed_digits(int(s), c) for s in scalars]
    sums = []
    for w in range(windows):
        buckets = [xyzz_inf(F) for _ in range(half)]
        for i in range(n):
            d = digits[i][w]
            if d == 0 or bases[i] is None:
                continue
            p = bases[i] if d > 0 else affine_neg(F, bases[i])
            buckets[abs(d) - 1] = xyzz_add_affine(F, buckets[abs(d) - 1], p)
        run, tot = xyzz_inf(F), xyzz_inf(F)
        for b in range(half - 1, -1, -1):
            run = xyzz_add(F, run, buckets[b])
            tot = xyzz_add(F, tot, run)
        sums.append(tot)
    acc = sums[-1]
    for w in range(windows - 2, -1, -1):
        for _ in range(c):
            acc = xyzz_double(F, acc) if not F.is_zero(acc[2]) else acc
        acc = xyzz_add(F, acc, sums[w])
    return xyzz_to_affine_point(F, acc)


def msm_naive(group: str, bases, scalars):
    F = FIELD[group]
    acc = None
    for p, s in zip(bases, scalars):
        acc = affine_add(F, acc, scalar_mul(F, p, int(s)))
    return acc


# ---------------------------------------------------------------- NTT

def ntt(values, inverse: bool = False):
    """X[k] = sum_i x[i] w^(ik) with w = root_of_unity(log_n); the inverse uses w^-1
    and includes the 1/n factor (src/ntt.rs:26-50). Natural order in and out."""
    a = [int(v) % R for v in values]
    n = len(a)
    log_n = n.bit_length() - 1
    assert 1 << log_n == n
    w = root_of_unity(log_n)
    if inverse:
        w = inv(w, R)
    # Decimation in frequency, bit-reversed result, then permute (src/shaders/ntt.wgsl).
    h = n // 2
    stage = 0
    while h >= 1:
        wstep = pow(w, 1 << stage, R)
        for start in range(0, n, 2 * h):
            tw = 1
            for j in range(start, start + h):
                x, y = a[j], a[j + h]
                a[j] = (x + y) % R
                a[j + h] = (x - y) * tw % R
                tw = tw * wstep % R
        h //= 2
        stage += 1
    out = [0] * n
    for i in range(n):
        out[int(format(i, f"0{log_n}b")[::-1], 2) if log_n else 0] = a[i]
    if inverse:
        ninv = inv(n, R)
        out = [x * ninv % R for x in out]
    return out


def ntt_direct(values, k: int, inverse: bool = False) -> int:
    """One output X[k] by Horner evaluation: O(n), for spot checks at large sizes."""
    n = len(values)
    w = root_of_unity(n.bit_length() - 1)
    if inverse:
        w = inv(w, R)
    x = pow(w, k, R)
    acc = 0
    for v in reversed(values):
        acc = (acc * x + int(v)) % R
    if inverse:
        acc = acc * inv(n, R) % R
    return acc


# ---------------------------------------------------------------- result conversion

def xyzz_words_to_affine(words, group: str = "G1", mont_r: int = MONT):
    """The library's XYZZ result words (Montgomery form, radix `mont_r`) -> affine point or
    None (src/msm.rs:345-373). Fq2 coordinates are (a, b) word pairs."""
    F = FIELD[group]
    rinv = inv(mont_r % Q, Q)
    coords = []
    if group == "G1":
        for i in range(4):
            coords.append(from_words32(words[8 * i: 8 * i + 8]) * rinv % Q)
    else:
        for i in range(4):
            a = from_words32(words[16 * i: 16 * i + 8]) * rinv % Q
            b = from_words32(words[16 * i + 8: 16 * i + 16]) * rinv % Q
            coords.append(Fq2(a, b))
    return xyzz_to_affine_point(F, tuple(coords))


def affine_words(group: str, p, mont_r: int = 1) -> list[int]:
    """Affine point -> memory words (x then y; Fq2 as a then b); infinity = all zeros.
    mont_r = 1 gives plain coordinates, 2^256 gives the snarkjs/ffjavascript form."""
    if group == "G1":
        if p is None:
            return [0] * 16
        return words32(p[0] * mont_r % Q) + words32(p[1] * mont_r % Q)
    if p is None:
        return [0] * 32
    out = []
    for c in (p[0], p[1]):
        out += words32(c.a * mont_r % Q) + words32(c.b * mont_r % Q)
    return out


def self_check() -> None:
    """Checks the oracle's own constants: both generators on their curves and of order r,
    the root of unity primitive, and Fq2 arithmetic consistent."""
    assert on_curve("G1", G1_GEN)
    g2 = (Fq2(*G2_GEN[0]), Fq2(*G2_GEN[1]))
    assert on_curve("G2", g2), "G2 generator is not on the twist y^2 = x^3 + 3/(9+u)"
    # [r]G = O: scalar_mul reduces k mod r, so test [r-1]G = -G instead.
    assert scalar_mul(_FqOps, G1_GEN, R - 1) == affine_neg(_FqOps, G1_GEN)
    assert scalar_mul(_Fq2Ops, g2, R - 1) == affine_neg(_Fq2Ops, g2)
    w = root_of_unity(28)
    assert pow(w, 1 << 28, R) == 1 and pow(w, 1 << 27, R) != 1


def g2_generator():
    return (Fq2(*G2_GEN[0]), Fq2(*G2_GEN[1]))


# ---------------------------------------------------------------- GLV split (G1)

def _cube_root(m: int) -> int:
    """The first g^((m-1)/3) != 1 over g = 2, 3, ...: a primitive cube root of unity mod m."""
    g = 2
    while pow(g, (m - 1) // 3, m) == 1:
        g += 1
    return pow(g, (m - 1) // 3, m)


def _glv_basis(lam: int):
    """Short vectors (a1, b1), (a2, b2) with a + b lam = 0 (mod R), by the extended Euclidean
    algorithm on (R, lam) (Guide to Elliptic Curve Cryptography, algorithm 3.74)."""
    import math
    rows = [(R, 0), (lam, 1)]
    while rows[-1][0] != 0:
        (r0, t0), (r1, t1) = rows[-2], rows[-1]
        q = r0 // r1
        rows.append((r0 - q * r1, t0 - q * t1))
    root = math.isqrt(R)
    ell = max(i for i, (r, _) in enumerate(rows) if r >= root)
    a1, b1 = rows[ell + 1][0], -rows[ell + 1][1]
    cand = [(rows[ell][0], -rows[ell][1]), (rows[ell + 2][0], -rows[ell + 2][1])]
    a2, b2 = min(cand, key=lambda v: v[0] * v[0] + v[1] * v[1])
    return a1, b1, a2, b2


_GLV = None


def glv_constants() -> dict:
    """beta (Fq), lambda (Fr) with (beta x, y) = lambda (x, y) on G1, the lattice basis and the
    fixed-point rounding constants g1 = round(2^256 b2 / r), g2 = round(2^256 (-b1) / r)."""
    global _GLV
    if _GLV is None:
        beta, lam0 = _cube_root(Q), _cube_root(R)
        probe = scalar_mul(_FqOps, G1_GEN, 0x1234567)
        lam = next(l for l in (lam0, lam0 * lam0 % R)
                   if scalar_mul(_FqOps, probe, l) == (beta * probe[0] % Q, probe[1]))
        a1, b1, a2, b2 = _glv_basis(lam)
        assert a1 * b2 - a2 * b1 == R
        rnd = lambda num: (2 * num * (1 << 256) + R) // (2 * R)
        _GLV = {"beta": beta, "lambda": lam, "a1": a1, "b1": b1, "a2": a2, "b2": b2,
                "g1": rnd(b2), "g2": rnd(-b1)}
    return _GLV


def glv_split(k: int) -> tuple[int, int]:
    """k (any 256-bit value, taken mod r) -> (k1, k2), signed, k = k1 + k2 lambda (mod r):
    c1 = floor((k g1 + 2^255) / 2^256), c2 = floor((k g2 + 2^255) / 2^256), k1 = k - c1 a1 -
    c2 a2, k2 = -c1 b1 - c2 b2."""
    g = glv_constants()
    k %= R
    c1 = (k * g["g1"] + (1 << 255)) >> 256
    c2 = (k * g["g2"] + (1 << 255)) >> 256
    return k - c1 * g["a1"] - c2 * g["a2"], -c1 * g["b1"] - c2 * g["b2"]
