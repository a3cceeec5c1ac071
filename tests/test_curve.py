"""Device point operations against the oracle, every special case included
(the reference's tests/curve.rs:57-87): P + Q (mixed), 2P, (P + Q) + 2P (full add)."""
import ctypes

import numpy as np
import pytest

from oracle import bn254
from zk_gpu._lib import check, lib, u32p

pytestmark = pytest.mark.gpu


def mont(x):
    return x * (1 << 256) % bn254.Q


def affine_mont_words(group, p):
    if p is None:
        return [0] * (16 if group == "G1" else 32)
    if group == "G1":
        return bn254.words32(mont(p[0])) + bn254.words32(mont(p[1]))
    return sum((bn254.words32(mont(c.a)) + bn254.words32(mont(c.b)) for c in (p[0], p[1])), [])


def from_xyzz(group, w):
    return bn254.xyzz_words_to_affine([int(v) for v in w], group)


@pytest.mark.parametrize("group", ["G1", "G2"])
def test_point_ops_match_the_oracle(gpu, group):
    F = bn254.FIELD[group]
    gen = bn254.G1_GEN if group == "G1" else bn254.g2_generator()
    rnd = np.random.default_rng(7 if group == "G1" else 8)
    pt = lambda: bn254.scalar_mul(F, gen, int(rnd.integers(1, 1 << 62)) * 0x1234567 + 99)
    p, q = pt(), pt()
    cases = [(p, q), (p, p), (p, bn254.affine_neg(F, p)), (None, q), (p, None), (None, None)]
    cases += [(pt(), pt()) for _ in range(20)]
    words = np.array([w for a, b in cases for w in affine_mont_words(group, a) + affine_mont_words(group, b)],
                     dtype=np.uint32)
    xw = 32 if group == "G1" else 64
    out = np.zeros(len(cases) * 3 * xw, dtype=np.uint32)
    check(lib().zkg_test_point_ops(gpu.handle, 1 if group == "G1" else 2, words.ctypes.data_as(u32p), len(cases),
                                   out.ctypes.data_as(u32p)))
    for i, (a, b) in enumerate(cases):
        got = lambda k: from_xyzz(group, out[(3 * i + k) * xw: (3 * i + k + 1) * xw])
        s = bn254.affine_add(F, a, b)
        d = bn254.affine_add(F, a, a)
        assert got(0) == s, f"case {i}: P + Q"
        assert got(1) == d, f"case {i}: 2P"
        assert got(2) == bn254.affine_add(F, s, d), f"case {i}: (P+Q) + 2P"
