"""The Groth16 quotient step on a coset (zkg_quotient, zkg_ntt_forward_quotient) against the
oracle: h_i = (a_i b_i - c_i) / (g^N - 1) over plain Fr values, alone and fused into the forward
transform of c (the pointwise products the reference leaves to callers, README.md:229-230)."""
import numpy as np
import pytest

from common import random_fr
from oracle import bn254, cpu
from zk_gpu import Ntt, ZkGpuError, quotient

pytestmark = pytest.mark.gpu
R = bn254.R


def words_to_ints(w):
    return [bn254.from_words32(w[8 * i: 8 * i + 8]) for i in range(w.size // 8)]


def h_ref(a, b, c, g, log_n):
    zinv = pow((pow(g, 1 << log_n, R) - 1) % R, R - 2, R)
    return np.array([x for ai, bi, ci in zip(words_to_ints(a), words_to_ints(b), words_to_ints(c))
                     for x in bn254.words32((ai * bi - ci) * zinv % R)], dtype=np.uint32)


@pytest.mark.parametrize("log_n", [10, 13])
def test_quotient_matches_oracle(gpu, log_n):
    n = 1 << log_n
    a, b, c = random_fr(800 + log_n, n), random_fr(801 + log_n, n), random_fr(802 + log_n, n)
    g = 7
    ab = gpu.buffer(a)
    quotient(gpu, ab, gpu.buffer(b), gpu.buffer(c), log_n, g)
    assert np.array_equal(gpu.read(ab, a.size), h_ref(a, b, c, g, log_n))


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("log_n", [10, 12, 15])
def test_forward_quotient_matches_oracle(gpu, log_n, form):
    """Every butterfly form: 2, 3 and 4 run the quotient in the transform's last pass, 0 and 1 after it."""
    n = 1 << log_n
    a, b, c = random_fr(810 + log_n, n), random_fr(811 + log_n, n), random_fr(812 + log_n, n)
    g = 5
    want = h_ref(a, b, cpu.ntt(c), g, log_n)
    ntt = Ntt(gpu, log_n)
    ntt.set_variant(form)
    data = gpu.buffer(c)
    ntt.forward_quotient(gpu, data, gpu.buffer(a), gpu.buffer(b), g)
    assert np.array_equal(gpu.read(data, c.size), want), (log_n, form)


def test_quotient_edge_values(gpu):
    """Zero, one and r - 1 entries, and a b = c (h = 0)."""
    log_n, n = 10, 1 << 10
    vals = [0, 1, R - 1, 2, R - 2]
    a = np.array([w for i in range(n) for w in bn254.words32(vals[i % 5])], dtype=np.uint32)
    b = np.array([w for i in range(n) for w in bn254.words32(vals[(i // 5) % 5])], dtype=np.uint32)
    c = np.array([w for i in range(n) for w in bn254.words32(vals[i % 5] * vals[(i // 5) % 5] % R if i % 3 else vals[(i // 25) % 5])],
                 dtype=np.uint32)
    ab = gpu.buffer(a)
    quotient(gpu, ab, gpu.buffer(b), gpu.buffer(c), log_n, 3)
    assert np.array_equal(gpu.read(ab, a.size), h_ref(a, b, c, 3, log_n))


def test_generator_of_the_subgroup_is_rejected(gpu):
    """g^N = 1 (g in H itself) makes the vanishing polynomial zero on the coset."""
    log_n = 10
    w = bn254.root_of_unity(log_n)
    buf = gpu.buffer(np.zeros(8 << log_n, dtype=np.uint32))
    with pytest.raises(ZkGpuError, match="g\\^N = 1"):
        quotient(gpu, buf, buf, buf, log_n, w)
    with pytest.raises(ZkGpuError, match="coset generator must be below r"):
        quotient(gpu, buf, buf, buf, log_n, R)
