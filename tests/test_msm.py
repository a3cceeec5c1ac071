"""G1 MSM against the oracle (tests/msm.rs:10-67), the property suite
(tests/properties.rs:150-431) and the full benchmark sizes through the identity
MSM([k_i]G, s) = [sum_i s_i k_i]G with bases built on the device."""
import os

import numpy as np
import pytest

from common import fr_words, gpu_msm, msm_ref, quick, random_fr, random_points
from oracle import bn254, cpu
from zk_gpu import Group, Msm, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.synthetic import generator_multiples, infinity_mask, scalar_distribution, uniform_scalars

pytestmark = pytest.mark.gpu
R = bn254.R


def check(gpu, bases, scalars, c, what, variant=None):
    """Both the plain windows and the default (the GLV split for G1, c <= 16)."""
    expected = msm_ref("G1", bases, scalars)
    for item_points in (1024, 7):
        for glv in (False, None):
            got = gpu_msm(gpu, bases, scalars, (c, item_points), variant=variant, glv=glv)
            assert np.array_equal(got, expected), (f"{what} (n = {scalars.size // 8}, c = {c}, item_points = "
                                                   f"{item_points}, variant = {variant}, glv = {glv})")


# Accumulation kernel forms checked by the edge-case suites: the default, and the G1 forms
# whose bucket arithmetic runs in double-precision limbs (their own special-case paths).
EDGE_VARIANTS = [None, 3, 4]


@pytest.mark.parametrize("variant", EDGE_VARIANTS)
def test_random_inputs(gpu, variant):
    for n, c in [(1000, 9), (4096, 10), (20000, 12), (100000, 14)]:
        check(gpu, random_points("G1", n, n), random_fr(n + 1, n), c, "random", variant)


@pytest.mark.parametrize("variant", EDGE_VARIANTS)
def test_edge_cases(gpu, variant):
    n, c = 3000, 10
    p = random_points("G1", 1, 1)
    rand = random_points("G1", 2, n)
    rand_s = random_fr(3, n)
    check(gpu, rand, fr_words([0] * n), c, "all-zero scalars", variant)
    check(gpu, rand, fr_words([1] * n), c, "all-one scalars (one huge bucket)", variant)
    check(gpu, rand, fr_words([R - 1] * n), c, "scalars = r - 1", variant)
    same = np.tile(p, n)
    check(gpu, same, rand_s, c, "same base everywhere (forces doublings)", variant)
    check(gpu, same, fr_words([5] * n), c, "same base, same scalar", variant)
    check(gpu, rand, fr_words(i % 7 for i in range(n)), c, "tiny scalars", variant)
    with_inf = rand.copy()
    with_inf[16 * 3: 16 * 4] = 0
    with_inf[16 * 100: 16 * 101] = 0
    check(gpu, with_inf, rand_s, c, "bases containing infinity", variant)
    negp = np.array(bn254.affine_words("G1", bn254.affine_neg(bn254._FqOps, (bn254.from_words32(p[:8]),
                                                                            bn254.from_words32(p[8:])))),
                    dtype=np.uint32)
    cancel = np.concatenate([p, negp, rand[:16 * 8]])
    cs = np.concatenate([rand_s[:8], rand_s[:8], np.zeros(64, dtype=np.uint32)])
    check(gpu, cancel, cs, c, "cancels to the point at infinity", variant)


def test_default_parameters(gpu):
    n = 1 << 17
    bases, scalars = random_points("G1", 30, n), random_fr(31, n)
    assert np.array_equal(gpu_msm(gpu, bases, scalars), msm_ref("G1", bases, scalars))


def add_affine(a, b):
    F = bn254._FqOps
    pa = None if not a.any() else (bn254.from_words32(a[:8]), bn254.from_words32(a[8:16]))
    pb = None if not b.any() else (bn254.from_words32(b[:8]), bn254.from_words32(b[8:16]))
    return np.array(bn254.affine_words("G1", bn254.affine_add(F, pa, pb)), dtype=np.uint32)


def scal(s: np.ndarray):
    return [bn254.from_words32(s[8 * i: 8 * i + 8]) for i in range(s.size // 8)]


def test_is_linear_in_the_scalars(gpu):
    n = 3000
    bases = random_points("G1", 10, n)
    s, t = random_fr(11, n), random_fr(12, n)
    sum_ = fr_words((a + b) % R for a, b in zip(scal(s), scal(t)))
    expected = add_affine(gpu_msm(gpu, bases, s), gpu_msm(gpu, bases, t))
    assert np.array_equal(gpu_msm(gpu, bases, sum_), expected), "MSM(s + t) != MSM(s) + MSM(t)"


def test_is_linear_in_the_bases(gpu):
    n = 3000
    p, q = random_points("G1", 13, n), random_points("G1", 14, n)
    s = random_fr(15, n)
    sum_ = np.concatenate([add_affine(p[16 * i: 16 * i + 16], q[16 * i: 16 * i + 16]) for i in range(n)])
    expected = add_affine(gpu_msm(gpu, p, s), gpu_msm(gpu, q, s))
    assert np.array_equal(gpu_msm(gpu, sum_, s), expected), "MSM(P + Q) != MSM(P) + MSM(Q)"


def test_scales_with_a_constant(gpu):
    n = 3000
    bases = random_points("G1", 16, n)
    s = random_fr(17, n)
    c = 0xABCDEF0123456789ABCDEF
    scaled = fr_words(x * c % R for x in scal(s))
    m = gpu_msm(gpu, bases, s)
    expected = np.array(bn254.affine_words("G1", bn254.scalar_mul(
        bn254._FqOps, (bn254.from_words32(m[:8]), bn254.from_words32(m[8:])), c)), dtype=np.uint32)
    assert np.array_equal(gpu_msm(gpu, bases, scaled), expected), "MSM(c * s) != c * MSM(s)"


def test_ignores_the_order_of_the_pairs(gpu):
    n = 5000
    bases, s = random_points("G1", 18, n), random_fr(19, n)
    order = np.random.default_rng(20).permutation(n)
    b2 = bases.reshape(n, 16)[order].reshape(-1)
    s2 = s.reshape(n, 8)[order].reshape(-1)
    assert np.array_equal(gpu_msm(gpu, b2, s2), gpu_msm(gpu, bases, s))


def test_tiny_inputs(gpu):
    for n in [1, 2, 3, 7, 17, 255, 256, 257, 1023, 1025]:
        bases, s = random_points("G1", 21 + n, n), random_fr(22 + n, n)
        want = msm_ref("G1", bases, s)
        for plan in [None, (9, 1024), (9, 1)]:
            assert np.array_equal(gpu_msm(gpu, bases, s, plan), want), f"n = {n}, plan = {plan}"


def test_bases_already_in_montgomery_form(gpu):
    for n in [1, 5, 300, 2000]:
        bases = random_points("G1", 40 + n, n)
        bases[16 * (n // 2): 16 * (n // 2) + 16] = 0
        s = random_fr(41 + n, n)
        buf = Msm.upload_bases_montgomery_256(gpu, cpu.fq_to_mont256(bases))
        msm = Msm(gpu, n, Msm.default_window(n))
        got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, buf, gpu.buffer(s)), 32)))
        assert np.array_equal(got, msm_ref("G1", bases, s)), f"n = {n}"


def test_huge_buckets(gpu):
    for n in [17, 300, 5000]:
        bases = random_points("G1", 50 + n, n)
        rnd = np.random.default_rng(n)
        same = fr_words([7] * n)
        ones = fr_words([1] * n)
        mostly = fr_words(int(v) if i % 50 == 0 else 3 for i, v in enumerate(rnd.integers(0, 1 << 62, size=n)))
        for scalars in (same, ones, mostly):
            want = msm_ref("G1", bases, scalars)
            for plan in [(9, 1), (10, 3), None]:
                assert np.array_equal(gpu_msm(gpu, bases, scalars, plan), want), f"n = {n}, plan = {plan}"


def test_nearly_empty_top_window(gpu):
    n = 20000
    bases, s = random_points("G1", 60, n), random_fr(61, n)
    want = msm_ref("G1", bases, s)
    for plan in [(14, 8), (14, 1), (11, 8)]:
        assert np.array_equal(gpu_msm(gpu, bases, s, plan), want), f"plan = {plan}"


def test_generator_multiples_2_18(gpu):
    """Big enough for many accumulate segments per bucket and several merge levels."""
    n = 1 << 18
    k = np.array([w for i in range(1, n + 1) for w in bn254.words32(i)], dtype=np.uint32)
    bases = cpu.generator_multiples("G1", k)
    s = random_fr(62, n)
    want = msm_ref("G1", bases, s)
    for plan in [None, (15, 8)]:
        assert np.array_equal(gpu_msm(gpu, bases, s, plan), want), f"plan = {plan}"


def boundary_scalars(c):
    out = [0, 1, R - 1, R - 2, R - (1 << c)]
    for j in range(1, -(-254 // c) + 1):
        for k in (c * j - 1, c * j):
            p = pow(2, k, R)
            out += [(p - 1) % R, p, (p + 1) % R]
    return out


def test_window_boundaries(gpu):
    for c in range(9, 17):
        vals = boundary_scalars(c) * 2
        s = fr_words(vals)
        bases = random_points("G1", 70 + c, len(vals))
        want = msm_ref("G1", bases, s)
        for item_points in (1024, 3):
            assert np.array_equal(gpu_msm(gpu, bases, s, (c, item_points)), want), f"c = {c}, items = {item_points}"


def test_result_does_not_depend_on_the_window_size(gpu):
    n = 6000
    bases, s = random_points("G1", 80, n), random_fr(81, n)
    want = msm_ref("G1", bases, s)
    for c in range(9, 21):
        assert np.array_equal(gpu_msm(gpu, bases, s, (c, 1024)), want), f"window size c = {c}"


def test_plan_can_be_reused(gpu):
    n = 4000
    bases = random_points("G1", 90, n)
    base_buf = Msm.upload_bases(gpu, bases)
    msm = Msm(gpu, n, 11)
    sets = [random_fr(91, n), fr_words([0] * n), fr_words([1] * n), random_fr(92, n)]
    for rnd in range(2):
        for i, s in enumerate(sets):
            out = msm.run(gpu, base_buf, gpu.buffer(s))
            got = affine_words(xyzz_to_affine(gpu.read(out, 32)))
            assert np.array_equal(got, msm_ref("G1", bases, s)), f"round {rnd}, scalar set {i}"


def fuzz_case(gpu, seed):
    rnd = np.random.default_rng(seed)
    n = int([rnd.integers(1, 64), rnd.integers(1, 1500), rnd.integers(1, 6000)][rnd.integers(0, 3)])
    c = int(rnd.integers(9, 17))
    item_points = int([1, 2, 5, 64, 1024][rnd.integers(0, 5)])
    scalar_kind = int(rnd.integers(0, 5))
    base_kind = int(rnd.integers(0, 3))
    pool = random_points("G1", seed * 3 + 1, 4).reshape(4, 16)
    fresh = random_points("G1", seed * 3 + 2, n).reshape(n, 16)
    if base_kind == 0:
        bases = fresh
    elif base_kind == 1:
        bases = pool[rnd.integers(0, 4, size=n)]
    else:
        bases = fresh.copy()
        bases[rnd.random(n) < 0.1] = 0
    if scalar_kind == 0:
        s = random_fr(seed * 3 + 3, n)
    elif scalar_kind == 1:
        s = fr_words(int(v) for v in rnd.integers(0, 16, size=n))
    elif scalar_kind == 2:
        s = random_fr(seed * 3 + 3, n).reshape(n, 8)
        s[rnd.random(n) < 0.9] = 0
        s = s.reshape(-1)
    elif scalar_kind == 3:
        s = fr_words(int(v) for v in rnd.integers(0, 1 << 63, size=n, dtype=np.uint64))
    else:
        s = fr_words([0, 1, R - 1][int(v)] for v in rnd.integers(0, 3, size=n))
    bases = np.ascontiguousarray(bases.reshape(-1))
    glv = bool(rnd.integers(0, 2))
    got = gpu_msm(gpu, bases, s, (c, item_points), glv=glv)
    assert np.array_equal(got, msm_ref("G1", bases, s)), (
        f"FUZZ FAILURE: rerun with ZK_GPU_FUZZ_SEED={seed} (n={n}, c={c}, item_points={item_points}, "
        f"scalars={scalar_kind}, bases={base_kind}, glv={glv})")


def fuzz_forms_case(gpu, seed):
    """One random edge-heavy MSM (G1, or G2 one time in four) through accumulation forms 1-4."""
    rnd = np.random.default_rng(seed)
    g = "G2" if int(rnd.integers(0, 4)) == 0 else "G1"
    group = Group.G2 if g == "G2" else Group.G1
    n = int([rnd.integers(1, 64), rnd.integers(1, 1500), rnd.integers(1, 5000)][rnd.integers(0, 3)])
    n = min(n, 1500) if g == "G2" else n
    c = int(rnd.integers(9, 17))
    item_points = int([1, 2, 5, 64, 1024][rnd.integers(0, 5)])
    aw = group.affine_words()
    pool = random_points(g, seed * 3 + 1, 4).reshape(4, aw)
    bases = random_points(g, seed * 3 + 2, n).reshape(n, aw)
    kind = int(rnd.integers(0, 3))
    if kind == 1:
        bases = pool[rnd.integers(0, 4, size=n)]  # repeats: doublings inside buckets
    elif kind == 2:
        bases = bases.copy()
        bases[rnd.random(n) < 0.1] = 0  # points at infinity
    sk = int(rnd.integers(0, 3))
    if sk == 0:
        s = random_fr(seed * 3 + 3, n)
    elif sk == 1:
        s = fr_words(int(v) for v in rnd.integers(0, 16, size=n))
    else:
        s = fr_words([0, 1, R - 1][int(v)] for v in rnd.integers(0, 3, size=n))
    bases = np.ascontiguousarray(bases.reshape(-1))
    want = msm_ref(g, bases, s)
    for variant in (1, 2, 3, 4):
        got = gpu_msm(gpu, bases, s, (c, item_points), group=group, variant=variant,
                      glv=bool(variant & 1) if g == "G1" else None)
        assert np.array_equal(got, want), (
            f"seed {seed}: {g} n={n} c={c} item_points={item_points} bases={kind} scalars={sk} form {variant}")


def test_fuzz_every_form(gpu):
    """Every accumulation form on the same random edge-heavy inputs (G1 and G2)."""
    for seed in range(5000, 5000 + (10 if quick() else 40)):
        fuzz_forms_case(gpu, seed)


def test_fuzz(gpu):
    if "ZK_GPU_FUZZ_SEED" in os.environ:
        return fuzz_case(gpu, int(os.environ["ZK_GPU_FUZZ_SEED"]))
    iters = int(os.environ.get("ZK_GPU_FUZZ_ITERS", 20 if quick() else 100))
    for seed in range(1000, 1000 + iters):
        fuzz_case(gpu, seed)


# ---------------------------------------------------------------- full sizes

def full_size_case(gpu, log_n, kind, c=None, inf_fraction=0.001, seed=0, variant=None, tuned=False, glv=None,
                   chunk=None):
    """Bases [k_i]G built on the device (0.1% at infinity: k_i = 0), read back in plain form and
    uploaded through Msm::upload_bases; the expected result is [sum_i s_i k_i]G. tuned: the plan
    (window, points per thread, form) comes from the autotuner on these inputs."""
    n = 1 << log_n
    k = uniform_scalars(n, 1000 + log_n + seed).reshape(n, 8)
    k[infinity_mask(n, inf_fraction, log_n + seed)] = 0
    k = k.reshape(-1)
    dev = generator_multiples(gpu, Group.G1, k)
    plain = gpu.read(dev, n * 16)
    dev.free()
    s = scalar_distribution(n, kind, 2000 + log_n + seed)
    c = c or Msm.default_window(n)
    base_buf, scalar_buf = Msm.upload_bases(gpu, plain), gpu.buffer(s)
    if tuned:
        from zk_gpu.autotune import tuned_msm
        msm = tuned_msm(gpu, Group.G1, n, base_buf, scalar_buf, reps=1)
        c, variant = msm.params()["c"], msm.params()["variant"]
    else:
        msm = Msm(gpu, n, c)
        if variant is not None:
            msm.set_variant(variant)
        if glv is not None:
            msm.set_glv(glv)
        if chunk is not None:
            msm.set_chunk(chunk)
    got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, base_buf, scalar_buf), 32)))
    gen = np.array(bn254.affine_words("G1", bn254.G1_GEN), dtype=np.uint32)
    want = cpu.scalar_mul("G1", gen, cpu.fr_dot(s, k))
    assert np.array_equal(got, want), f"G1 MSM 2^{log_n} ({kind}, c = {c}, variant = {variant}, glv = {glv}) wrong"
    # spot check the device-built bases against the CPU
    for i in (0, 1, n - 1):
        assert np.array_equal(plain[16 * i: 16 * i + 16], cpu.generator_multiples("G1", k[8 * i: 8 * i + 8]))


@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"])
@pytest.mark.parametrize("log_n", [18, 20, 22])
def test_full_size_distributions(gpu, log_n, kind):
    full_size_case(gpu, log_n, kind, glv=False)  # the plain windows (GLV: tests/test_glv.py)


@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"] if not quick() else ["uniform"])
def test_full_size_2_24(gpu, kind):
    full_size_case(gpu, 24, kind, glv=False)


@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"])
@pytest.mark.parametrize("log_n", [18, 20, 22])
def test_full_size_autotuned(gpu, log_n, kind, tmp_path, monkeypatch):
    """The same cases with the autotuned window, points per thread and form."""
    monkeypatch.setenv("ZK_GPU_TUNE_CACHE", str(tmp_path / "tune.json"))
    full_size_case(gpu, log_n, kind, tuned=True)


def test_full_size_in_passes(gpu):
    """A 2^22 run in passes of 2^20 and of 3 x 10^5 points (a short last pass), GLV and plain."""
    full_size_case(gpu, 22, "uniform", chunk=1 << 20)
    full_size_case(gpu, 22, "r-1", glv=False, chunk=300000)


def test_full_size_other_window(gpu):
    full_size_case(gpu, 20, "uniform", c=13)
    full_size_case(gpu, 20, "r-1", c=18)


@pytest.mark.parametrize("kind", ["uniform", "sparse", "r-1"])
@pytest.mark.parametrize("variant", [3, 4])
def test_full_size_double_precision_forms(gpu, variant, kind):
    full_size_case(gpu, 22, kind, variant=variant)
    full_size_case(gpu, 18, kind, c=16, variant=variant)


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_accumulation_variants_agree(gpu, variant):
    """Every form of the accumulation kernel (inlined / out-of-line integer field products,
    double-precision limbs)."""
    for n, c, items, kind in [(20000, 12, None, "uniform"), (5000, 10, 3, "r-1"), (3000, 9, 1, "sparse")]:
        bases = random_points("G1", 900 + n, n)
        s = scalar_distribution(n, kind, 901 + n)
        msm = Msm.with_item_points(gpu, n, c, items) if items else Msm(gpu, n, c)
        msm.set_variant(variant)
        assert msm.params()["variant"] == variant
        got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, Msm.upload_bases(gpu, bases), gpu.buffer(s)), 32)))
        assert np.array_equal(got, msm_ref("G1", bases, s)), (n, c, items, kind, variant)


def test_autotuned_plan_is_exact(gpu, tmp_path, monkeypatch):
    from zk_gpu.autotune import search_msm, tuned_msm
    monkeypatch.setenv("ZK_GPU_TUNE_CACHE", str(tmp_path / "tune.json"))
    n = 1 << 14
    bases = random_points("G1", 950, n)
    s = random_fr(951, n)
    bb, sb = Msm.upload_bases(gpu, bases), gpu.buffer(s)
    results = search_msm(gpu, Group.G1, n, bb, sb, reps=1)
    assert results and results == sorted(results, key=lambda r: r["ms"])
    assert {r["variant"] for r in results} == {1, 2, 3, 4}
    assert {r["glv"] for r in results} == {0, 1}
    msm = tuned_msm(gpu, Group.G1, n, bb, sb, reps=1)
    again = tuned_msm(gpu, Group.G1, n, bb, sb, reps=1)  # from the cache
    assert msm.params() == again.params()
    got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, bb, sb), 32)))
    assert np.array_equal(got, msm_ref("G1", bases, s))


@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_sort_aggregation_modes_agree(gpu, mode, form):
    """The counting sort's warp aggregation modes (every group / first lane's group / none) on
    inputs that put many lanes of a warp into one slot and on uniform ones, in both sort forms
    (atomic scatter, ranked placement)."""
    n, c = 20000, 12
    bases = random_points("G1", 960, n)
    cases = [("uniform", scalar_distribution(n, "uniform", 961)), ("sparse", scalar_distribution(n, "sparse", 962)),
             ("r-1", scalar_distribution(n, "r-1", 963)), ("all ones", fr_words([1] * n)),
             ("alternating", fr_words([5 if i % 2 else R - 5 for i in range(n)]))]
    for name, s in cases:
        for items in (None, 3):
            msm = Msm.with_item_points(gpu, n, c, items) if items else Msm(gpu, n, c)
            msm.set_sort(mode)
            msm.set_sort_form(form)
            got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, Msm.upload_bases(gpu, bases), gpu.buffer(s)), 32)))
            assert np.array_equal(got, msm_ref("G1", bases, s)), (name, items, mode, form)


@pytest.mark.parametrize("form", [0, 1])
def test_slots_beyond_the_rank_field(gpu, form):
    """More than 2^16 entries in one slot (every scalar 1, or r - 1: all points in one bucket of
    window 0), in both sort forms: ranks past 16 bits place correctly."""
    n = (1 << 17) + 3
    bases = random_points("G1", 970, n)
    for s in (fr_words([1] * n), fr_words([R - 1] * (n - 5) + [2, 3, 0, 7, R - 2])):
        msm = Msm(gpu, n, 16)
        msm.set_sort_form(form)
        got = affine_words(xyzz_to_affine(gpu.read(msm.run(gpu, Msm.upload_bases(gpu, bases), gpu.buffer(s)), 32)))
        assert np.array_equal(got, msm_ref("G1", bases, s)), form


@pytest.mark.parametrize("group", ["G1", "G2"])
def test_fixed_base_tables(gpu, group):
    """A plan in fixed-base mode over the table of 2^(c w) P_i gives the plain MSM's point: every
    window's digits in one set of buckets, no combination. Window sizes 9..16, points at infinity,
    and scalars 0, 1, r - 1 and window-boundary values (whose signed digits carry into the next
    window) beside uniform ones; table rows spot-checked against the oracle."""
    grp = Group.G1 if group == "G1" else Group.G2
    n = 1500
    bases = random_points(group, 980, n)
    aw = grp.affine_words()
    bases[: aw * 3] = 0  # three points at infinity
    base_buf = Msm.upload_bases(gpu, bases)
    special = [0, 1, R - 1, (1 << 15) - 1, 1 << 15, (1 << 16) + (1 << 15), R - (1 << 20)]
    for c in (9, 11, 13, 16):
        table = Msm.fixed_base_table(gpu, grp, base_buf, n, c)
        windows = (255 + c - 1) // c
        if c == 11:  # rows: 2^(c w) P_i for a few (w, i)
            words = gpu.read(table, windows * n * aw)
            for w, i in ((0, 5), (1, 7), (windows - 1, 9)):
                row = words[(w * n + i) * aw: (w * n + i + 1) * aw]
                want = cpu.scalar_mul(group, bases[i * aw: (i + 1) * aw], np.array(bn254.words32(pow(2, c * w, R)),
                                                                                   dtype=np.uint32))
                assert np.array_equal(cpu.fq_to_mont256(want), row), (w, i)
        for seed in (0, 1):
            s = random_fr(990 + c + seed, n).reshape(n, 8)
            if seed:
                for j, v in enumerate(special):
                    s[j] = bn254.words32(v)
            s = s.reshape(-1)
            msm = Msm.for_group(gpu, grp, n, c)
            msm.set_fixed_base(True)
            words = gpu.read(msm.run(gpu, table, gpu.buffer(s)), grp.xyzz_words())
            conv = xyzz_to_affine if grp == Group.G1 else xyzz_to_affine_g2
            assert np.array_equal(affine_words(conv(words), grp), msm_ref(group, bases, s)), (group, c, seed)


def test_fixed_base_checks(gpu):
    n = 64
    bases = Msm.upload_bases(gpu, random_points("G1", 985, n))
    msm = Msm(gpu, n, 17)
    with pytest.raises(Exception, match="c <= 16"):
        msm.set_fixed_base(True)
    msm = Msm(gpu, n, 12)
    msm.set_fixed_base(True)
    with pytest.raises(Exception, match="bases buffer holds"):
        msm.run(gpu, bases, gpu.buffer(random_fr(986, n)))  # the key itself, not its table


@pytest.mark.parametrize("group", ["G1", "G2"])
def test_passes(gpu, group):
    """Runs split into passes of at most `chunk` points (zkg_msm_set_chunk) give the one-pass
    point for every slice size, including one point per pass and a short last pass; the plan's
    stage profile sums the passes; a fixed-base plan runs in one pass."""
    grp = Group.G1 if group == "G1" else Group.G2
    n = 5000 if group == "G1" else 1200
    bases = random_points(group, 1900, n)
    bases[: grp.affine_words() * 2] = 0  # two points at infinity
    s = random_fr(1901, n).reshape(n, 8)
    s[5] = bn254.words32(R - 1)
    s[6] = 0
    s = s.reshape(-1)
    want = msm_ref(group, bases, s)
    base_buf, scalar_buf = Msm.upload_bases(gpu, bases), gpu.buffer(s)
    conv = xyzz_to_affine if grp == Group.G1 else xyzz_to_affine_g2
    chunks = [1, 7, 1000, n // 2, n - 1, n, 10 * n, 0] if group == "G1" else [333, n - 1, 0]
    for glv in ((False, True) if group == "G1" else (False,)):
        msm = Msm.for_group(gpu, grp, n, 11)
        msm.set_glv(glv)
        assert msm.passes() == (n, 1)
        for ch in chunks:
            msm.set_chunk(ch)
            per = min(ch or n, n)
            assert msm.passes() == (per, -(-n // per)), (ch, msm.passes())
            for _ in range(2):  # the scratch of every pass is reused
                got = affine_words(conv(gpu.read(msm.run(gpu, base_buf, scalar_buf), grp.xyzz_words())), grp)
                assert np.array_equal(got, want), (group, glv, ch)
    msm = Msm.for_group(gpu, grp, n, 11)
    msm.set_chunk(1000)
    stages = msm.profile(gpu, base_buf, scalar_buf)
    assert len(stages) == 8 and all(ms >= 0 for _, ms in stages)
    got = affine_words(conv(gpu.read(msm.run(gpu, base_buf, scalar_buf), grp.xyzz_words())), grp)
    assert np.array_equal(got, want)
    msm.set_fixed_base(True)  # one pass: the table's rows are n points apart
    assert msm.passes() == (n, 1)
    with pytest.raises(Exception, match="runs in one pass"):
        msm.set_chunk(100)
