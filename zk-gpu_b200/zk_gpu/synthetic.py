"""Seeded synthetic inputs with the shapes of the benchmark configurations: uniform Fr scalars
in [0, r), skewed scalar mixes, and proving-key-like bases [k_i]G built on the device.

Scalars: 8 LE u32 words each, uniform in [0, r) by rejection (the top word is drawn in
[0, r >> 224] and the rare draws >= r are redrawn). Bases: [k_i]G for the standard generator
of G1 (1, 2) or G2, computed by zkg_generator_multiples on the GPU (a 2^24-point key takes
well under a second there; the same points on the CPU take minutes).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib
from .gpu import Buffer, Gpu
from .group import Group
from .host import FR

_R_WORDS = np.array([(FR >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)


def _below_r(words: np.ndarray) -> np.ndarray:
    """Row mask: 8-word little-endian value < r."""
    lt = np.zeros(words.shape[0], dtype=bool)
    eq = np.ones(words.shape[0], dtype=bool)
    for i in range(7, -1, -1):
        lt |= eq & (words[:, i] < _R_WORDS[i])
        eq &= words[:, i] == _R_WORDS[i]
    return lt


def uniform_scalars(n: int, seed: int) -> np.ndarray:
    """n uniform elements of [0, r) as an (n*8,) uint32 array."""
    rng = np.random.default_rng(seed)
    out = rng.integers(0, 1 << 32, size=(n, 8), dtype=np.uint32)
    out[:, 7] = rng.integers(0, int(_R_WORDS[7]) + 1, size=n, dtype=np.uint32)
    bad = ~_below_r(out)
    while bad.any():
        k = int(bad.sum())
        redo = rng.integers(0, 1 << 32, size=(k, 8), dtype=np.uint32)
        redo[:, 7] = rng.integers(0, int(_R_WORDS[7]) + 1, size=k, dtype=np.uint32)
        out[bad] = redo
        bad = ~_below_r(out)
    return out.reshape(-1)


def small_scalars(n: int, seed: int, bits: int = 64) -> np.ndarray:
    """n uniform values below 2^bits (bits <= 64)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 8), dtype=np.uint32)
    v = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * 2 + rng.integers(0, 2, size=n, dtype=np.uint64)
    if bits < 64:
        v &= np.uint64((1 << bits) - 1)
    out[:, 0] = (v & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    out[:, 1] = (v >> np.uint64(32)).astype(np.uint32)
    return out.reshape(-1)


R_MINUS_1 = np.array([((FR - 1) >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)


def scalar_distribution(n: int, kind: str, seed: int) -> np.ndarray:
    """The three scalar mixes of the MSM configurations:
    'uniform'  uniform in [0, r);
    'sparse'   30% zero, 30% below 2^64, the rest uniform;
    'r-1'      5% equal to r - 1, the rest uniform."""
    s = uniform_scalars(n, seed).reshape(n, 8)
    rng = np.random.default_rng(seed ^ 0x5EED)
    if kind == "uniform":
        pass
    elif kind == "sparse":
        u = rng.random(n)
        s[u < 0.3] = 0
        mid = (u >= 0.3) & (u < 0.6)
        s[mid] = small_scalars(int(mid.sum()), seed + 1).reshape(-1, 8)
    elif kind == "r-1":
        s[rng.random(n) < 0.05] = R_MINUS_1
    else:
        raise ValueError(f"unknown scalar distribution {kind!r}")
    return s.reshape(-1)


def generator_multiples(gpu: Gpu, group: Group, k: np.ndarray, mont256: bool = False) -> Buffer:
    """Device buffer of [k_i]G (affine, plain or Montgomery-2^256 coordinates)."""
    k = np.ascontiguousarray(k, dtype=np.uint32)
    n = k.size // 8
    kbuf = gpu.buffer(k)
    out = gpu.empty_buffer(n * Group(group).affine_words())
    check(lib().zkg_generator_multiples(gpu.handle, int(group), kbuf.handle, n, int(mont256), out.handle))
    return out


def infinity_mask(n: int, fraction: float, seed: int) -> np.ndarray:
    """Seeded positions of the bases set to infinity ((0, 0)): k_i = 0 there."""
    rng = np.random.default_rng(seed ^ 0x1F1F)
    return rng.random(n) < fraction
