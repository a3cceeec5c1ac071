"""NTT against the oracle and its mathematical properties (tests/ntt.rs:9-34,
tests/properties.rs:25-138), plus the full benchmark sizes through size-independent checks."""
import numpy as np
import pytest

from common import fr_words, gpu_ntt, quick, random_fr
from oracle import bn254, cpu
from zk_gpu import Ntt, ZkGpuError

pytestmark = pytest.mark.gpu
R = bn254.R


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 16, 18, 20, 22])
def test_matches_oracle(gpu, log_n):
    x = random_fr(100 + log_n, 1 << log_n)
    ntt = Ntt(gpu, log_n)
    buf = gpu.buffer(x)
    ntt.forward(gpu, buf)
    got = gpu.read(buf, x.size)
    assert np.array_equal(got, cpu.ntt(x)), f"forward NTT mismatch at log_n={log_n}"
    ntt.inverse(gpu, buf)
    assert np.array_equal(gpu.read(buf, x.size), x), f"inverse NTT did not restore the input at log_n={log_n}"


@pytest.mark.parametrize("form", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("log_n", [10, 11, 13, 15, 17, 21])
def test_every_form_matches_oracle(gpu, log_n, form):
    """Each butterfly form: 0 integer, 1 FP64 with table twiddles, 2 / 3 FP64 with staged
    twiddles (one / two butterflies per thread step), 4 radix-4 with staged twiddles; sizes with
    one tile, even and odd stage counts per pass."""
    x = random_fr(340 + log_n, 1 << log_n)
    ntt = Ntt(gpu, log_n)
    ntt.set_variant(form)
    assert ntt.params()["variant"] == form
    want = cpu.ntt(x)
    assert np.array_equal(gpu_ntt(gpu, ntt, x), want), f"log_n={log_n} form={form}"
    assert np.array_equal(gpu_ntt(gpu, ntt, want, inverse=True), x), f"log_n={log_n} form={form}"


@pytest.mark.parametrize("log_n", [10, 11, 13, 16, 20])
def test_integer_form_matches_oracle(gpu, log_n):
    """The integer butterfly form (variant 0) beside the default double-precision one (which
    every other test of this file runs)."""
    x = random_fr(300 + log_n, 1 << log_n)
    ntt = Ntt(gpu, log_n)
    ntt.set_variant(0)
    assert ntt.params()["variant"] == 0
    assert np.array_equal(gpu_ntt(gpu, ntt, x), cpu.ntt(x)), f"log_n={log_n}"
    assert np.array_equal(gpu_ntt(gpu, ntt, cpu.ntt(x), inverse=True), x), f"log_n={log_n}"


@pytest.mark.parametrize("log_n", [24, 26] if not quick() else [24])
def test_full_size_matches_oracle(gpu, log_n):
    """At the benchmark sizes, every output: the forward transform equals the multi-threaded C
    oracle's element for element, the inverse of an oracle-made spectrum equals the oracle's
    inverse (a wrong root used consistently in both directions would pass a round trip, not
    this), and inverse(forward(x)) == x. Sampled O(n) evaluations X[k] tie the oracle itself to
    the definition at this size."""
    n = 1 << log_n
    x = random_fr(7 + log_n, n)
    want = cpu.ntt(x)
    ntt = Ntt(gpu, log_n)
    buf = gpu.buffer(x)
    ntt.forward(gpu, buf)
    y = gpu.read(buf, x.size)
    bad = np.flatnonzero((y != want).reshape(n, 8).any(axis=1))
    assert bad.size == 0, f"{bad.size} forward outputs differ at log_n={log_n}, first at {bad[:4]}"
    for k in [0, 1, n - 1, int(np.random.default_rng(log_n).integers(0, n))]:
        assert np.array_equal(want[8 * k: 8 * k + 8], cpu.ntt_eval(x, k)), f"oracle X[{k}] at log_n={log_n}"
    ntt.inverse(gpu, buf)
    assert np.array_equal(gpu.read(buf, x.size), x)
    del y
    spectrum = random_fr(17 + log_n, n)
    want_inv = cpu.ntt(spectrum, inverse=True)
    buf.write(spectrum)
    ntt.inverse(gpu, buf)
    got_inv = gpu.read(buf, x.size)
    bad = np.flatnonzero((got_inv != want_inv).reshape(n, 8).any(axis=1))
    assert bad.size == 0, f"{bad.size} inverse outputs differ at log_n={log_n}, first at {bad[:4]}"


def test_delta_is_a_power_sequence(gpu):
    for log_n in (10, 11, 13):
        n = 1 << log_n
        ntt = Ntt(gpu, log_n)
        w = bn254.root_of_unity(log_n)
        for k in [0, 1, 2, 511, 512, n - 1]:
            delta = np.zeros(8 * n, dtype=np.uint32)
            delta[8 * k] = 1
            want = fr_words(pow(w, j * k, R) for j in range(n))
            assert np.array_equal(gpu_ntt(gpu, ntt, delta), want), f"NTT of delta_{k} wrong at log_n={log_n}"
        c = 123456789
        want = np.zeros(8 * n, dtype=np.uint32)
        want[:8] = bn254.words32(c * n % R)
        assert np.array_equal(gpu_ntt(gpu, ntt, fr_words([c] * n)), want)


def test_is_linear(gpu):
    for log_n in (10, 12, 14):
        n = 1 << log_n
        ntt = Ntt(gpu, log_n)
        a, b = random_fr(1, n), random_fr(2, n)
        c = 0x1234567890ABCDEF1234567
        av = [bn254.from_words32(a[8 * i: 8 * i + 8]) for i in range(n)]
        bv = [bn254.from_words32(b[8 * i: 8 * i + 8]) for i in range(n)]
        comb = fr_words((x * c + y) % R for x, y in zip(av, bv))
        fa, fb = gpu_ntt(gpu, ntt, a), gpu_ntt(gpu, ntt, b)
        fav = [bn254.from_words32(fa[8 * i: 8 * i + 8]) for i in range(n)]
        fbv = [bn254.from_words32(fb[8 * i: 8 * i + 8]) for i in range(n)]
        want = fr_words((x * c + y) % R for x, y in zip(fav, fbv))
        assert np.array_equal(gpu_ntt(gpu, ntt, comb), want), f"linearity failed at log_n={log_n}"


def test_convolution_theorem(gpu):
    n = 1 << 10
    ntt = Ntt(gpu, 10)
    a, b = random_fr(3, n), random_fr(4, n)
    av = [bn254.from_words32(a[8 * i: 8 * i + 8]) for i in range(n)]
    bv = [bn254.from_words32(b[8 * i: 8 * i + 8]) for i in range(n)]
    expected = [0] * n
    for i, x in enumerate(av):
        if x:
            for j, y in enumerate(bv):
                expected[(i + j) % n] += x * y
    expected = fr_words(v % R for v in expected)
    fa, fb = gpu_ntt(gpu, ntt, a), gpu_ntt(gpu, ntt, b)
    prod = fr_words(bn254.from_words32(fa[8 * i: 8 * i + 8]) * bn254.from_words32(fb[8 * i: 8 * i + 8]) % R
                    for i in range(n))
    assert np.array_equal(gpu_ntt(gpu, ntt, prod, inverse=True), expected), "convolution theorem failed"


def test_round_trips_in_both_directions(gpu):
    for log_n in (10, 15, 18):
        ntt = Ntt(gpu, log_n)
        x = random_fr(5 + log_n, 1 << log_n)
        assert np.array_equal(gpu_ntt(gpu, ntt, gpu_ntt(gpu, ntt, x), inverse=True), x)
        assert np.array_equal(gpu_ntt(gpu, ntt, gpu_ntt(gpu, ntt, x, inverse=True)), x)


def test_extreme_values(gpu):
    log_n = 12
    n = 1 << log_n
    ntt = Ntt(gpu, log_n)
    rnd = np.random.default_rng(4)
    mixed = fr_words([0, 1, R - 1][int(i)] for i in rnd.integers(0, 3, size=n))
    for name, inp in [("zeros", fr_words([0] * n)), ("ones", fr_words([1] * n)), ("r-1", fr_words([R - 1] * n)),
                      ("mixed", mixed)]:
        got = gpu_ntt(gpu, ntt, inp)
        assert np.array_equal(got, cpu.ntt(inp)), f"extreme input '{name}' wrong"
        assert np.array_equal(gpu_ntt(gpu, ntt, got, inverse=True), inp), f"'{name}' does not round-trip"


def test_plan_can_be_reused(gpu):
    log_n = 13
    n = 1 << log_n
    ntt = Ntt(gpu, log_n)
    inputs = [random_fr(50 + i, n) for i in range(4)]
    first = [gpu_ntt(gpu, ntt, x) for x in inputs]
    for i in reversed(range(4)):
        assert np.array_equal(gpu_ntt(gpu, ntt, inputs[i]), first[i]), f"second run of input {i} differs"
    assert np.array_equal(gpu_ntt(gpu, Ntt(gpu, log_n), inputs[0]), first[0])


COSET_G = 7  # Fr's multiplicative generator, the usual coset offset of a Groth16 witness map


@pytest.mark.parametrize("log_n", [10, 14, 20])
def test_coset_shift_matches_oracle(gpu, log_n):
    from zk_gpu import CosetShift
    x = random_fr(300 + log_n, 1 << log_n)
    buf = gpu.buffer(x)
    CosetShift(gpu, log_n, COSET_G).shift(gpu, buf)
    g = np.array(bn254.words32(COSET_G), dtype=np.uint32)
    assert np.array_equal(gpu.read(buf, x.size), cpu.coset_shift(x, g))


def test_coset_evaluation_chain(gpu):
    """inverse -> coset shift -> forward (evaluations on the coset g*H), as the witness map does."""
    from zk_gpu import CosetShift
    log_n = 16
    x = random_fr(400, 1 << log_n)
    ntt = Ntt(gpu, log_n)
    buf = gpu.buffer(x)
    ntt.inverse(gpu, buf)
    CosetShift(gpu, log_n, COSET_G).shift(gpu, buf)
    ntt.forward(gpu, buf)
    g = np.array(bn254.words32(COSET_G), dtype=np.uint32)
    want = cpu.ntt(cpu.coset_shift(cpu.ntt(x, True), g))
    assert np.array_equal(gpu.read(buf, x.size), want)
    # and back: inverse, shift by g^-1, forward returns the input
    ntt.inverse(gpu, buf)
    CosetShift(gpu, log_n, pow(COSET_G, R - 2, R)).shift(gpu, buf)
    ntt.forward(gpu, buf)
    assert np.array_equal(gpu.read(buf, x.size), x)


@pytest.mark.parametrize("log_n", [10, 11, 12, 17, 20])
def test_inverse_with_fused_coset_shift(gpu, log_n):
    """inverse_coset (the shift in the inverse's last pass) gives the words of inverse followed
    by the shift kernel, for one-tile and multi-pass sizes, in both butterfly forms, for two
    shifts on one plan (their tables are kept apart)."""
    from zk_gpu import CosetShift
    x = random_fr(500 + log_n, 1 << log_n)
    g = np.array(bn254.words32(COSET_G), dtype=np.uint32)
    ginv = np.array(bn254.words32(pow(COSET_G, R - 2, R)), dtype=np.uint32)
    want = cpu.coset_shift(cpu.ntt(x, True), g)
    want_inv = cpu.coset_shift(cpu.ntt(x, True), ginv)
    ntt = Ntt(gpu, log_n)
    shift, unshift = CosetShift(gpu, log_n, COSET_G), CosetShift(gpu, log_n, pow(COSET_G, R - 2, R))
    for variant in (0, 1, 2, 3, 4):
        ntt.set_variant(variant)
        for sh, expect in ((shift, want), (unshift, want_inv), (shift, want)):
            buf = gpu.buffer(x)
            ntt.inverse_coset(gpu, buf, sh)
            assert np.array_equal(gpu.read(buf, x.size), expect), f"variant {variant}"
    # the unfused calls agree word for word
    buf = gpu.buffer(x)
    ntt.set_variant(0)
    ntt.inverse(gpu, buf)
    shift.shift(gpu, buf)
    assert np.array_equal(gpu.read(buf, x.size), want)


def test_fused_coset_shift_checks_sizes(gpu):
    from zk_gpu import CosetShift
    ntt = Ntt(gpu, 12)
    buf = gpu.empty_buffer(8 << 12)
    with pytest.raises(ZkGpuError, match="coset shift of 2\\^11 elements on a 2\\^12 transform"):
        ntt.inverse_coset(gpu, buf, CosetShift(gpu, 11, COSET_G))


def test_coset_rejects_bad_generator(gpu):
    from zk_gpu import CosetShift, ZkGpuError
    with pytest.raises(ZkGpuError, match="below r"):
        CosetShift(gpu, 12, R)


def test_every_pass_split_is_exact(gpu, tmp_path, monkeypatch):
    from zk_gpu.autotune import tuned_ntt
    log_n = 20
    x = random_fr(500, 1 << log_n)
    want = cpu.ntt(x)
    for variant, top in ((0, 11), (1, 10), (2, 10), (3, 10), (4, 10)):
        for s in range(6, top + 1):
            ntt = Ntt(gpu, log_n)
            ntt.set_variant(variant)
            ntt.set_max_stages(s)
            p = ntt.params()
            assert (p["variant"], p["max_stages"]) == (variant, s)
            assert np.array_equal(gpu_ntt(gpu, ntt, x), want), f"variant {variant}, max_stages = {s}"
            assert np.array_equal(gpu_ntt(gpu, ntt, want, inverse=True), x), f"variant {variant}, max_stages = {s}"
        with pytest.raises(ZkGpuError):
            ntt.set_max_stages(top + 1)
    monkeypatch.setenv("ZK_GPU_TUNE_CACHE", str(tmp_path / "tune.json"))
    buf = gpu.buffer(x)
    ntt = tuned_ntt(gpu, log_n, buf, reps=1)
    assert np.array_equal(gpu_ntt(gpu, ntt, x), want)


def test_plans_of_different_sizes_interleave(gpu):
    """A small plan made after a large one does not shrink what the large one's passes may use
    (a per-kernel launch limit): both forms, run in turn."""
    big_x, small_x = random_fr(600, 1 << 16), random_fr(601, 1 << 10)
    big = Ntt(gpu, 16)
    small = Ntt(gpu, 10)
    for variant in (0, 1, 4, 2, 0, 3):
        big.set_variant(variant)
        small.set_variant(variant)
        assert np.array_equal(gpu_ntt(gpu, big, big_x), cpu.ntt(big_x)), f"variant {variant}"
        assert np.array_equal(gpu_ntt(gpu, small, small_x), cpu.ntt(small_x)), f"variant {variant}"
        Ntt(gpu, 10)  # another small plan between runs
