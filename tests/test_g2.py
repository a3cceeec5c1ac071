"""The G2 MSM (points over Fq2) against the oracle (tests/g2.rs:50-148), plus full sizes via
MSM([k_i]G2, s) = [sum s_i k_i]G2."""
import numpy as np
import pytest

from common import fr_words, gpu_msm, msm_ref, random_fr, random_points
from oracle import bn254, cpu
from zk_gpu import Group, Msm, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.synthetic import generator_multiples, uniform_scalars

pytestmark = pytest.mark.gpu
R = bn254.R
G2 = Group.G2


def test_g2_msm_matches_oracle(gpu):
    for n in [1, 2, 3, 17, 255, 1000, 4000]:
        bases, s = random_points("G2", 21 + n, n), random_fr(22 + n, n)
        want = msm_ref("G2", bases, s)
        for c, items in [(13, None), (9, 1), (10, 64)]:
            assert np.array_equal(gpu_msm(gpu, bases, s, (c, items), G2), want), f"n = {n}, c = {c}"


def test_g2_special_scalars_and_infinity(gpu):
    n = 600
    bases = random_points("G2", 30, n).reshape(n, 32)
    bases[7] = 0
    bases[8] = bases[9]
    bases = bases.reshape(-1)
    vals = [bn254.from_words32(random_fr(31, n)[8 * i: 8 * i + 8]) for i in range(n)]
    vals[0], vals[1], vals[2], vals[3], vals[8], vals[9] = 0, 1, R - 1, pow(2, 200, R), 5, 5
    s = fr_words(vals)
    assert np.array_equal(gpu_msm(gpu, bases, s, (10, None), G2), msm_ref("G2", bases, s))
    assert not gpu_msm(gpu, bases, fr_words([0] * n), (10, None), G2).any()
    p = bases[20 * 32: 21 * 32]
    x = 0x1234567890ABCDEF
    assert not gpu_msm(gpu, np.concatenate([p, p]), fr_words([x, R - x]), (9, None), G2).any()


def test_g2_bases_in_ffjavascript_montgomery_form(gpu):
    n = 500
    bases = random_points("G2", 40, n).reshape(n, 32)
    bases[3] = 0
    bases = bases.reshape(-1)
    s = random_fr(41, n)
    buf = Msm.upload_bases_montgomery_256(gpu, cpu.fq_to_mont256(bases))
    msm = Msm.for_group(gpu, G2, n, 10)
    got = affine_words(xyzz_to_affine_g2(gpu.read(msm.run(gpu, buf, gpu.buffer(s)), 64)), G2)
    assert np.array_equal(got, msm_ref("G2", bases, s))


def test_g2_huge_buckets(gpu):
    for n in [300, 3000]:
        bases = random_points("G2", 50 + n, n)
        rnd = np.random.default_rng(n)
        same = fr_words([7] * n)
        mostly = fr_words(int(v) if i % 50 == 0 else 3 for i, v in enumerate(rnd.integers(0, 1 << 62, size=n)))
        for s in (same, mostly):
            want = msm_ref("G2", bases, s)
            for c, items in [(9, 1), (10, 3), (13, None)]:
                assert np.array_equal(gpu_msm(gpu, bases, s, (c, items), G2), want), f"n = {n}, c = {c}"


def test_g2_2_16(gpu):
    n = 1 << 16
    k = np.array([w for i in range(1, n + 1) for w in bn254.words32(i)], dtype=np.uint32)
    bases = cpu.generator_multiples("G2", k)
    s = random_fr(60, n)
    assert np.array_equal(gpu_msm(gpu, bases, s, (13, None), G2), msm_ref("G2", bases, s))


@pytest.mark.parametrize("log_n", [18, 20, 22])
def test_g2_full_size_montgomery_upload(gpu, log_n):
    n = 1 << log_n
    k = uniform_scalars(n, 3000 + log_n)
    dev = generator_multiples(gpu, G2, k, mont256=True)
    mont = gpu.read(dev, n * 32)
    dev.free()
    s = uniform_scalars(n, 4000 + log_n)
    buf = Msm.upload_bases_montgomery_256(gpu, mont)
    msm = Msm.for_group(gpu, G2, n, Msm.default_window(n))
    got = affine_words(xyzz_to_affine_g2(gpu.read(msm.run(gpu, buf, gpu.buffer(s)), 64)), G2)
    gen = np.array(bn254.affine_words("G2", bn254.g2_generator()), dtype=np.uint32)
    assert np.array_equal(got, cpu.scalar_mul("G2", gen, cpu.fr_dot(s, k)))
    for i in (0, n - 1):
        assert np.array_equal(mont[32 * i: 32 * i + 32],
                              cpu.generator_multiples("G2", k[8 * i: 8 * i + 8], mont256=True))


@pytest.mark.parametrize("variant", [1, 3, 4])
def test_g2_accumulation_forms_agree(gpu, variant):
    """Integer (one product per call) and double-precision (two / one per call) accumulation on
    random inputs, repeated bases (doublings) and cancelling pairs."""
    n = 2000
    bases = random_points("G2", 70, n).reshape(n, 32)
    bases[5] = 0
    bases[10:20] = bases[9]
    bases = bases.reshape(-1)
    p = bases[40 * 32: 41 * 32]
    cases = [random_fr(71, n), fr_words([7] * n), fr_words(i % 5 for i in range(n))]
    for s in cases:
        want = msm_ref("G2", bases, s)
        for c, items in [(10, None), (9, 3)]:
            assert np.array_equal(gpu_msm(gpu, bases, s, (c, items), G2, variant=variant), want), (variant, c, items)
    x = 0x1234567890ABCDEF
    cancel = np.concatenate([p, p, bases[:32 * 6]])
    cs = np.concatenate([fr_words([x, R - x]), random_fr(72, 6)])
    assert np.array_equal(gpu_msm(gpu, cancel, cs, (9, None), G2, variant=variant), msm_ref("G2", cancel, cs))


@pytest.mark.parametrize("variant", [3, 4])
def test_g2_full_size_double_precision(gpu, variant):
    log_n = 20
    n = 1 << log_n
    k = uniform_scalars(n, 3100 + log_n)
    dev = generator_multiples(gpu, G2, k, mont256=True)
    s = uniform_scalars(n, 4100 + log_n)
    msm = Msm.for_group(gpu, G2, n, Msm.default_window(n))
    msm.set_variant(variant)
    got = affine_words(xyzz_to_affine_g2(gpu.read(msm.run(gpu, dev, gpu.buffer(s)), 64)), G2)
    gen = np.array(bn254.affine_words("G2", bn254.g2_generator()), dtype=np.uint32)
    assert np.array_equal(got, cpu.scalar_mul("G2", gen, cpu.fr_dot(s, k)))
