"""The C-ABI library without a GPU: it loads, exports every symbol include/zkg.h declares, and
its host-only functions (default window, XYZZ -> affine conversion) are right."""
import os
import re

import numpy as np
import pytest

from oracle import bn254
import zk_gpu
from zk_gpu import Msm, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu._lib import LIB_PATH, SIGNATURES, lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "zkg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zkg_[a-z0-9_]+)\s*\(", text)))


def test_library_is_built_in_tree():
    assert os.path.exists(LIB_PATH), "run `make -C zk-gpu_b200` (or __graft_entry__.build())"


def test_every_declared_symbol_is_exported_and_bound():
    L = lib()
    names = declared_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), f"{name} declared in include/zkg.h but not exported"
        assert name in SIGNATURES, f"{name} has no ctypes signature"


def test_default_window_matches_reference_formula():
    for n in [0, 1, 2, 1000, 1 << 10, 1 << 16, 1 << 17, 1 << 20, 1 << 21, 1 << 22, 1 << 24, 1 << 26]:
        want = min(max(max(n, 1).bit_length() - 1 - 5, 11), 16)
        assert Msm.default_window(n) == want, n


def _mont(x):
    return x * (1 << 256) % bn254.Q


def test_xyzz_to_affine_on_the_host():
    rnd = np.random.default_rng(4)
    for trial in range(5):
        k = int(rnd.integers(1, 1 << 62))
        x, y = bn254.scalar_mul(bn254._FqOps, bn254.G1_GEN, k)
        z = int(rnd.integers(1, 1 << 62))
        zz, zzz = z * z % bn254.Q, z * z * z % bn254.Q
        words = (bn254.words32(_mont(x * zz)) + bn254.words32(_mont(y * zzz)) + bn254.words32(_mont(zz))
                 + bn254.words32(_mont(zzz)))
        got = xyzz_to_affine(np.array(words, dtype=np.uint32))
        assert got is not None
        assert zk_gpu.host.from_u64s(got[0]) == x and zk_gpu.host.from_u64s(got[1]) == y
    assert xyzz_to_affine(np.zeros(32, dtype=np.uint32)) is None


def test_xyzz_to_affine_g2_on_the_host():
    g2 = bn254.g2_generator()
    p = bn254.scalar_mul(bn254._Fq2Ops, g2, 123456789)
    z = bn254.Fq2(5, 11)
    zz = z * z
    zzz = zz * z
    coords = [p[0] * zz, p[1] * zzz, zz, zzz]
    words = []
    for c in coords:
        words += bn254.words32(_mont(c.a)) + bn254.words32(_mont(c.b))
    got = xyzz_to_affine_g2(np.array(words, dtype=np.uint32))
    f = zk_gpu.host.from_u64s
    assert (f(got[0][0]), f(got[0][1]), f(got[1][0]), f(got[1][1])) == (p[0].a, p[0].b, p[1].a, p[1].b)
    assert xyzz_to_affine_g2(np.zeros(64, dtype=np.uint32)) is None


def test_host_helpers_follow_the_reference():
    h = zk_gpu.host
    assert h.root_of_unity(28) == bn254.root_of_unity(28)
    assert h.from_words32(h.words32(h.FQ - 1)) == h.FQ - 1
    assert h.from_montgomery(_mont(12345), h.FQ) == 12345


def test_no_gpu_is_reported_not_hidden():
    """Without a CUDA device, making a context fails with ZKG_ENODEV instead of falling back."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(zk_gpu.ZkGpuError) as e:
        zk_gpu.Gpu()
    assert e.value.code == 6 and "no GPU adapter" in str(e.value)
