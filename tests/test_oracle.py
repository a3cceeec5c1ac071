"""The oracle itself, pinned before it is trusted (CPU only).

Both restatements (the big-integer one in oracle/bn254.py and the C one in oracle/zkg_oracle.c)
must reproduce the reference's golden vectors (tests/golden/*.json, ffjavascript 0.3.1) bit for
bit, agree with each other on G1 and G2 inputs, and agree with naive sums of scalar
multiplications (the reference's tests/properties.rs:433-442 guard of the guard).
"""
import hashlib
import os
import random

import numpy as np
import pytest

from common import GOLDEN, golden_msm_cases, golden_ntt_cases
from oracle import bn254, cpu

PINNED = {
    "ntt.json": "7cd9ee744f1538f8e7d032ff1073cbc81b1b2a9ecfad564ef7fc78d39fe599f0",
    "msm.json": "cfff456b4002ebe4f6e1b925d9988703ec29d79d2cb380d2b436e7a11c42deb6",
}


def test_golden_files_are_the_references():
    for name, digest in PINNED.items():
        with open(os.path.join(GOLDEN, name), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == digest, name


def test_oracle_constants():
    bn254.self_check()


def _points(words, group="G1"):
    aw = 16 if group == "G1" else 32
    out = []
    for i in range(words.size // aw):
        w = [int(v) for v in words[aw * i: aw * i + aw]]
        if not any(w):
            out.append(None)
        elif group == "G1":
            out.append((bn254.from_words32(w[0:8]), bn254.from_words32(w[8:16])))
        else:
            out.append((bn254.Fq2(bn254.from_words32(w[0:8]), bn254.from_words32(w[8:16])),
                        bn254.Fq2(bn254.from_words32(w[16:24]), bn254.from_words32(w[24:32]))))
    return out


def _scalars(words):
    return [bn254.from_words32(words[8 * i: 8 * i + 8]) for i in range(words.size // 8)]


@pytest.mark.parametrize("case", golden_ntt_cases(), ids=lambda c: f"{c[0]}-{'inv' if c[1] else 'fwd'}")
def test_ntt_oracles_match_golden(case):
    log_n, inverse, inp, out = case
    assert np.array_equal(cpu.ntt(inp, inverse), out)
    got = bn254.ntt(_scalars(inp), inverse)
    assert got == _scalars(out)
    for k in (0, 1, 7, (1 << log_n) - 1):
        assert np.array_equal(cpu.ntt_eval(inp, k, inverse), out[8 * k: 8 * k + 8])


@pytest.mark.parametrize("case", golden_msm_cases(), ids=lambda c: c[0])
def test_msm_oracles_match_golden(case):
    name, bases, scalars, result = case
    for c in (0, 4, 9, 12, 16):
        assert np.array_equal(cpu.msm("G1", bases, scalars, c=c), result), (name, c)
    assert np.array_equal(cpu.msm("G1", cpu.fq_to_mont256(bases), scalars, mont256=True), result)
    got = bn254.msm_pippenger("G1", _points(bases), _scalars(scalars), c=10)
    assert bn254.affine_words("G1", got) == [int(v) for v in result]


def test_msm_oracle_is_a_sum_of_scalar_multiplications():
    rnd = random.Random(18)
    for group in ("G1", "G2"):
        ks = [rnd.randrange(bn254.R) for _ in range(12)]
        bases = cpu.generator_multiples(group, np.array([w for k in ks for w in bn254.words32(k)], dtype=np.uint32))
        ss = [rnd.randrange(bn254.R) for _ in range(12)]
        scalars = np.array([w for s in ss for w in bn254.words32(s)], dtype=np.uint32)
        naive = bn254.msm_naive(group, _points(bases, group), ss)
        assert [int(v) for v in cpu.msm(group, bases, scalars)] == bn254.affine_words(group, naive)
        zero = np.zeros_like(scalars)
        assert not cpu.msm(group, bases, zero).any()


def test_generator_multiples_match_python():
    rnd = random.Random(3)
    ks = [0, 1, 2, bn254.R - 1, bn254.R, (1 << 256) - 1] + [rnd.randrange(1 << 256) for _ in range(6)]
    kw = np.array([w for k in ks for w in bn254.words32(k)], dtype=np.uint32)
    g1 = cpu.generator_multiples("G1", kw)
    g2 = cpu.generator_multiples("G2", kw)
    for i, k in enumerate(ks):
        assert [int(v) for v in g1[16 * i: 16 * i + 16]] == bn254.affine_words(
            "G1", bn254.scalar_mul(bn254._FqOps, bn254.G1_GEN, k))
        assert [int(v) for v in g2[32 * i: 32 * i + 32]] == bn254.affine_words(
            "G2", bn254.scalar_mul(bn254._Fq2Ops, bn254.g2_generator(), k))


def test_msm_identity_used_at_full_size():
    """MSM([k_i]G, s) = [sum s_i k_i]G: the size-independent check of the large runs."""
    rnd = np.random.default_rng(5)
    from zk_gpu.synthetic import uniform_scalars
    k = uniform_scalars(3000, 1)
    s = uniform_scalars(3000, 2)
    for group in ("G1", "G2"):
        bases = cpu.generator_multiples(group, k)
        gen = cpu.generator_multiples(group, np.array(bn254.words32(1), dtype=np.uint32))
        expect = cpu.scalar_mul(group, gen, cpu.fr_dot(s, k))
        assert np.array_equal(cpu.msm(group, bases, s), expect)
    del rnd


def test_g2_oracles_agree():
    rnd = random.Random(21)
    n = 17
    ks = [rnd.randrange(bn254.R) for _ in range(n)]
    bases = cpu.generator_multiples("G2", np.array([w for k in ks for w in bn254.words32(k)], dtype=np.uint32))
    ss = [rnd.randrange(bn254.R) for _ in range(n)]
    scalars = np.array([w for s in ss for w in bn254.words32(s)], dtype=np.uint32)
    want = bn254.affine_words("G2", bn254.msm_pippenger("G2", _points(bases, "G2"), ss, c=9))
    for c in (0, 9, 13):
        assert [int(v) for v in cpu.msm("G2", bases, scalars, c=c)] == want
    mont = cpu.fq_to_mont256(bases)
    assert [int(v) for v in cpu.msm("G2", mont, scalars, mont256=True)] == want


def test_ntt_oracle_round_trip_and_coset():
    from zk_gpu.synthetic import uniform_scalars
    x = uniform_scalars(1 << 12, 9)
    assert np.array_equal(cpu.ntt(cpu.ntt(x), True), x)
    g = np.array(bn254.words32(7), dtype=np.uint32)
    shifted = cpu.coset_shift(x, g)
    vals = [bn254.from_words32(x[8 * i: 8 * i + 8]) for i in range(8)]
    for i in range(8):
        assert bn254.from_words32(shifted[8 * i: 8 * i + 8]) == vals[i] * pow(7, i, bn254.R) % bn254.R
