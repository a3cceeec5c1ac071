"""GLV splitting of the G1 MSM (zkg_msm_set_glv). The reference has no GLV code (it names GLV as
its next step, README.md:223-224), so these tests hold the split to the oracle's restatement
(oracle/bn254.py glv_split, constants derived there from q and r alone) and every GLV MSM to
the plain MSM's result: the reference's own suites (tests/msm.rs:10-67, tests/properties.rs)
run with the split on."""
import numpy as np
import pytest

from common import fr_words, golden_msm_cases, gpu_msm, msm_ref, quick, random_fr, random_points
from oracle import bn254
from zk_gpu import Group, Msm, ZkGpuError, lib
from zk_gpu._lib import check as check_status

R, Q = bn254.R, bn254.Q


def edge_scalars(rnd) -> list[int]:
    g = bn254.glv_constants()
    lam = g["lambda"]
    out = [0, 1, 2, R - 1, R - 2, R, R + 1, 2 * R - 1, (1 << 256) - 1, (1 << 255), (1 << 254) - 1,
           lam, R - lam, lam * lam % R, (R - 1) // 2, (R + 1) // 2, 1 << 127, (1 << 128) - 1]
    # scalars where c1 or c2 sits next to a rounding boundary: k ~ (j + 1/2) r / b2
    for _ in range(200):
        j = int(rnd.integers(0, 1 << 62)) * int(rnd.integers(1, 1 << 62))
        for b in (g["b2"], -g["b1"]):
            k = ((2 * j + 1) * R) // (2 * b) % R
            out += [k, (k + 1) % R, (k - 1) % R]
    return out


def raw_words(values) -> np.ndarray:
    return np.array([w for v in values for w in bn254.words32(int(v))], dtype=np.uint32)


# ---------------------------------------------------------------- the split (CPU)

def test_constants_define_the_endomorphism():
    g = bn254.glv_constants()
    beta, lam = g["beta"], g["lambda"]
    assert beta != 1 and pow(beta, 3, Q) == 1
    assert (lam * lam + lam + 1) % R == 0
    F = bn254._FqOps
    for k in (1, 7, 0x1234567890abcdef, R - 5):
        p = bn254.scalar_mul(F, bn254.G1_GEN, k)
        assert bn254.scalar_mul(F, p, lam) == (beta * p[0] % Q, p[1])
    for a, b in ((g["a1"], g["b1"]), (g["a2"], g["b2"])):
        assert (a + b * lam) % R == 0
    assert g["a1"] * g["b2"] - g["a2"] * g["b1"] == R
    assert abs(g["a1"]) < 1 << 127 and abs(g["b2"]) < 1 << 127
    assert abs(g["a2"]) < 1 << 64 and abs(g["b1"]) < 1 << 64


def test_split_is_exact_and_short():
    """k = k1 + k2 lambda (mod r) and |k1|, |k2| < 5/8 (a1 + a2) < 2^126.2 < 2^127, the bound the
    device's ceil(128 / c) windows rest on."""
    g = bn254.glv_constants()
    bound = (5 * (abs(g["a1"]) + abs(g["a2"]))) // 8 + 1
    assert bound < 1 << 127
    rnd = np.random.default_rng(7)
    ks = edge_scalars(rnd) + [int.from_bytes(rnd.bytes(32), "little") for _ in range(20000)]
    for k in ks:
        k1, k2 = bn254.glv_split(k)
        assert (k1 + k2 * g["lambda"] - k) % R == 0, hex(k)
        assert abs(k1) < bound and abs(k2) < bound, hex(k)


def test_window_widths():
    """The GLV windows (glv_window_pos / glv_window_width in msm_kernels.cuh): W = ceil(128 / c)
    windows cover bits 0..127 exactly, none wider than c (their digits fit the plan's 2^(c-1)
    buckets), and the top one is wide enough that a half below 2^126.2 leaves its digit below
    half its range (no carry out of the last window)."""
    for c in range(9, 17):
        w = -(-128 // c)
        widths = [128 // w + (1 if i < 128 % w else 0) for i in range(w)]
        assert sum(widths) == 128 and max(widths) <= c, c
        top = widths[-1]
        assert 2 ** (126.2 - (128 - top)) + 1 < 2 ** (top - 1), c


# ---------------------------------------------------------------- the split (GPU)

@pytest.mark.gpu
def test_device_split_matches_the_oracle(gpu):
    rnd = np.random.default_rng(11)
    ks = edge_scalars(rnd) + [int.from_bytes(rnd.bytes(32), "little") for _ in range(20000)]
    words = raw_words(ks)
    out = np.zeros(10 * len(ks), dtype=np.uint32)
    check_status(lib().zkg_test_glv_split(gpu.handle, words.ctypes.data_as(lib().zkg_test_glv_split.argtypes[1]),
                                          len(ks), out.ctypes.data_as(lib().zkg_test_glv_split.argtypes[3])))
    out = out.reshape(-1, 10)
    for i, k in enumerate(ks):
        k1, k2 = bn254.glv_split(k)
        got1 = bn254.from_words32(list(out[i, 0:4]) + [0] * 4) * (-1 if out[i, 8] else 1)
        got2 = bn254.from_words32(list(out[i, 4:8]) + [0] * 4) * (-1 if out[i, 9] else 1)
        assert (got1, got2) == (k1, k2), f"scalar {hex(k)}"


# ---------------------------------------------------------------- GLV MSMs against the oracle

def check(gpu, bases, scalars, c, what, variant=None):
    expected = msm_ref("G1", bases, scalars)
    for item_points in (1024, 7):
        got = gpu_msm(gpu, bases, scalars, (c, item_points), variant=variant, glv=True)
        assert np.array_equal(got, expected), \
            f"{what} (n = {scalars.size // 8}, c = {c}, item_points = {item_points}, variant = {variant}, GLV)"


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [None, 1, 2, 3, 4])
def test_random_inputs(gpu, variant):
    for n, c in [(1000, 9), (4096, 10), (20000, 12), (100000, 14), (3000, 16)]:
        check(gpu, random_points("G1", n, n), random_fr(n + 1, n), c, "random", variant)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [None, 3, 4])
def test_edge_cases(gpu, variant):
    n, c = 3000, 10
    p = random_points("G1", 1, 1)
    rand = random_points("G1", 2, n)
    rand_s = random_fr(3, n)
    check(gpu, rand, fr_words([0] * n), c, "all-zero scalars", variant)
    check(gpu, rand, fr_words([1] * n), c, "all-one scalars", variant)
    check(gpu, rand, fr_words([R - 1] * n), c, "scalars = r - 1", variant)
    lam = bn254.glv_constants()["lambda"]
    check(gpu, rand, fr_words([lam] * n), c, "scalars = lambda (k1 = 0, k2 = 1)", variant)
    same = np.tile(p, n)
    check(gpu, same, rand_s, c, "same base everywhere (forces doublings)", variant)
    check(gpu, same, fr_words([lam, 1, R - lam] * (n // 3)), c, "P, phi(P) and -phi(P) meet in buckets",
          variant)
    with_inf = rand.copy()
    with_inf[16 * 3: 16 * 4] = 0
    with_inf[16 * 100: 16 * 101] = 0
    check(gpu, with_inf, rand_s, c, "bases containing infinity", variant)
    rnd = np.random.default_rng(5)
    ks = edge_scalars(rnd)
    ks = [k % R for k in ks]
    check(gpu, random_points("G1", 4, len(ks)), fr_words(ks), 11, "split-boundary scalars", variant)


@pytest.mark.gpu
def test_golden_vectors(gpu):
    """The reference's golden MSMs (tests/golden/msm.json, ffjavascript) with the split on."""
    for name, bases, scalars, result in golden_msm_cases():
        n = scalars.size // 8
        for c in (9, 12, 16):
            got = gpu_msm(gpu, bases, scalars, (c, 7), glv=True)
            assert np.array_equal(got, result), f"MSM '{name}' (n = {n}, c = {c}, GLV) differs from ffjavascript"


def fuzz_case(gpu, seed):
    rnd = np.random.default_rng(seed)
    n = int([rnd.integers(1, 64), rnd.integers(1, 1500), rnd.integers(1, 6000)][rnd.integers(0, 3)])
    c = int(rnd.integers(9, 17))
    item_points = int([1, 2, 5, 64, 1024][rnd.integers(0, 5)])
    variant = [None, 1, 2, 3, 4][int(rnd.integers(0, 5))]
    pool = random_points("G1", seed * 3 + 1, 4).reshape(4, 16)
    bases = random_points("G1", seed * 3 + 2, n).reshape(n, 16)
    kind = int(rnd.integers(0, 3))
    if kind == 1:
        bases = pool[rnd.integers(0, 4, size=n)]
    elif kind == 2:
        bases = bases.copy()
        bases[rnd.random(n) < 0.1] = 0
    sk = int(rnd.integers(0, 4))
    lam = bn254.glv_constants()["lambda"]
    if sk == 0:
        s = random_fr(seed * 3 + 3, n)
    elif sk == 1:
        s = fr_words(int(v) for v in rnd.integers(0, 16, size=n))
    elif sk == 2:
        s = fr_words([0, 1, R - 1, lam, R - lam][int(v)] for v in rnd.integers(0, 5, size=n))
    else:
        s = fr_words(int(v) << 120 for v in rnd.integers(0, 1 << 62, size=n, dtype=np.uint64))
    bases = np.ascontiguousarray(bases.reshape(-1))
    got = gpu_msm(gpu, bases, s, (c, item_points), variant=variant, glv=True)
    assert np.array_equal(got, msm_ref("G1", bases, s)), (
        f"seed {seed}: n={n} c={c} item_points={item_points} variant={variant} bases={kind} scalars={sk}")


@pytest.mark.gpu
def test_fuzz(gpu):
    for seed in range(7000, 7000 + (20 if quick() else 60)):
        fuzz_case(gpu, seed)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"])
@pytest.mark.parametrize("log_n", [18, 20, 22])
def test_full_size_distributions(gpu, log_n, kind):
    from test_msm import full_size_case
    full_size_case(gpu, log_n, kind, glv=True)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"] if not quick() else ["uniform"])
def test_full_size_2_24(gpu, kind):
    from test_msm import full_size_case
    full_size_case(gpu, 24, kind, glv=True)


@pytest.mark.gpu
def test_switching_and_checks(gpu):
    n = 5000
    bases, scalars = random_points("G1", 40, n), random_fr(41, n)
    want = msm_ref("G1", bases, scalars)
    msm = Msm(gpu, n, 12)
    assert msm.windows() == (11, True)  # the G1 default where it applies
    base_buf, scalar_buf = Msm.upload_bases(gpu, bases), gpu.buffer(scalars)
    from zk_gpu import xyzz_to_affine
    from zk_gpu.msm import affine_words
    for glv, windows in ((False, 22), (True, 11), (False, 22), (True, 11)):
        msm.set_glv(glv)
        assert msm.windows() == (windows, glv)
        got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, base_buf, scalar_buf), 32)))
        assert np.array_equal(got, want), f"GLV {glv}"
    assert Msm.for_group(gpu, Group.G2, 1024, 10).windows() == (26, False)
    assert Msm(gpu, 1024, 17).windows() == (15, False)
    with pytest.raises(ZkGpuError, match="GLV splitting is for G1"):
        Msm.for_group(gpu, Group.G2, 1024, 10).set_glv(True)
    with pytest.raises(ZkGpuError, match=r"GLV splitting needs a window size c <= 16, got 17"):
        Msm(gpu, 1024, 17).set_glv(True)
    msm.set_fixed_base(True)  # switches GLV off: a table's rows are the plain windows
    assert msm.windows() == (22, False)
    with pytest.raises(ZkGpuError, match="do not combine"):
        msm.set_glv(True)
