"""msm::Msm and the XYZZ -> affine conversions (src/msm.rs:25-387) over zkg_msm."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import StageTime, check, lib, u32p, u64p, vp
from .gpu import Buffer, Gpu, as_words
from .group import Group


class Msm:
    """A reusable plan for MSMs of `n` points in `group` with window size `c`
    (Msm::for_group, src/msm.rs:95-180)."""

    def __init__(self, gpu: Gpu, n: int, c: int, *, group: Group = Group.G1, item_points: int | None = None):
        h = vp()
        check(lib().zkg_msm_new(gpu.handle, int(group), n, c, item_points or 0, ctypes.byref(h)))
        self._h = h.value
        self._gpu = gpu
        self._group = Group(group)
        self.n = n
        self.c = c

    @staticmethod
    def default_window(n: int) -> int:
        """Msm::default_window (src/msm.rs:78-80)."""
        return lib().zkg_msm_default_window(n)

    @classmethod
    def new(cls, gpu: Gpu, n: int, c: int) -> "Msm":
        return cls(gpu, n, c)

    @classmethod
    def with_item_points(cls, gpu: Gpu, n: int, c: int, item_points: int) -> "Msm":
        return cls(gpu, n, c, item_points=item_points)

    @classmethod
    def for_group(cls, gpu: Gpu, group: Group, n: int, c: int, item_points: int | None = None) -> "Msm":
        return cls(gpu, n, c, group=group, item_points=item_points)

    @staticmethod
    def upload_bases(gpu: Gpu, plain_xy) -> Buffer:
        """Msm::upload_bases: plain affine coordinates -> device Montgomery form."""
        w = as_words(plain_xy)
        h = vp()
        check(lib().zkg_msm_upload_bases(gpu.handle, w.ctypes.data_as(u32p), w.size, ctypes.byref(h)))
        return Buffer(gpu, h.value)

    @staticmethod
    def upload_bases_montgomery_256(gpu: Gpu, xy) -> Buffer:
        """Msm::upload_bases_montgomery_256: coordinates already times 2^256 mod q."""
        w = as_words(xy)
        h = vp()
        check(lib().zkg_msm_upload_bases_montgomery_256(gpu.handle, w.ctypes.data_as(u32p), w.size,
                                                        ctypes.byref(h)))
        return Buffer(gpu, h.value)

    def group(self) -> Group:
        return self._group

    def set_variant(self, variant: int) -> None:
        """Accumulation kernel form: 0 inlined field products, 1 out-of-line (smaller code),
        2 out-of-line two at a time; 3 / 4 double-precision limbs, two / one product per call.
        Defaults: G1 4 (plain windows: 3 below 2^26 (window, point) entries and 4 from there),
        G2 2."""
        check(lib().zkg_msm_set_variant(self._h, variant))

    def set_sort(self, mode: int) -> None:
        """Counting-pass warp aggregation: 0 every group of equal slots, 1 the first lane's
        group, 2 none, 3 the first equal neighbour pair's group."""
        check(lib().zkg_msm_set_sort(self._h, mode))

    def set_fixed_base(self, enable: bool = True) -> None:
        """Runs take a fixed-base table (Msm.fixed_base_table) as their bases: one set of buckets
        for every window and no combination doublings; the same result as the plain MSM."""
        check(lib().zkg_msm_set_fixed_base(self._h, int(enable)))

    @staticmethod
    def fixed_base_table(gpu: Gpu, group: Group, bases: Buffer, n: int, c: int) -> Buffer:
        """Rows w = 0..ceil(255/c)-1 of 2^(c w) P_i for the n resident bases."""
        h = vp()
        check(lib().zkg_msm_fixed_base_table(gpu.handle, int(group), bases.handle, n, c, ctypes.byref(h)))
        return Buffer(gpu, h.value)

    def set_chunk(self, points: int) -> None:
        """Run in passes of at most `points` points (0: the largest the 32-bit entry indices
        allow); bounds the plan's scratch memory. The result does not change."""
        check(lib().zkg_msm_set_chunk(self._h, points))

    def passes(self) -> tuple[int, int]:
        """(points per pass, passes per run)."""
        ch, ps = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().zkg_msm_passes(self._h, ctypes.byref(ch), ctypes.byref(ps)))
        return ch.value, ps.value

    def set_glv(self, enable: bool = True) -> None:
        """G1: split every scalar as k1 + k2 lambda (mod r) and run over P_i and phi(P_i) with
        ceil(128 / c) windows; the same result as the plain MSM."""
        check(lib().zkg_msm_set_glv(self._h, int(enable)))

    def windows(self) -> tuple[int, bool]:
        """(window count, GLV on)."""
        w, g = ctypes.c_uint32(), ctypes.c_int()
        check(lib().zkg_msm_windows(self._h, ctypes.byref(w), ctypes.byref(g)))
        return w.value, bool(g.value)

    def set_sort_form(self, form: int) -> None:
        """Counting sort: 0 scatter through atomic cursors, 1 ranked placement window by window
        (default for c <= 16)."""
        check(lib().zkg_msm_set_sort_form(self._h, form))

    def params(self) -> dict:
        c, items, var = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_int()
        check(lib().zkg_msm_params(self._h, ctypes.byref(c), ctypes.byref(items), ctypes.byref(var)))
        windows, glv = self.windows()
        return {"c": c.value, "item_points": items.value, "variant": var.value, "windows": windows, "glv": glv}

    def run(self, gpu: Gpu, bases: Buffer, scalars: Buffer) -> Buffer:
        """Msm::run: queue sum(scalars[i] * bases[i]); returns the plan's XYZZ result buffer
        (borrowed: overwritten by the next run)."""
        out = vp()
        check(lib().zkg_msm_run(self._h, bases.handle, scalars.handle, ctypes.byref(out)))
        return Buffer(gpu, out.value, owned=False)

    def profile(self, gpu: Gpu, bases: Buffer, scalars: Buffer) -> list[tuple[str, float]]:
        """Msm::profile: (stage, milliseconds) per stage, device-timed."""
        arr = (StageTime * 32)()
        count = ctypes.c_size_t()
        check(lib().zkg_msm_profile(self._h, bases.handle, scalars.handle, arr, 32, ctypes.byref(count)))
        return [(arr[i].stage.decode(), arr[i].ms) for i in range(count.value)]

    def close(self) -> None:
        if self._h:
            lib().zkg_msm_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def xyzz_to_affine(words):
    """xyzz_to_affine (src/msm.rs:345-354): 32 result words -> ([u64;4], [u64;4]) plain
    affine coordinates, or None for the point at infinity."""
    w = as_words(words)
    assert w.size >= 32
    x = (ctypes.c_uint64 * 4)()
    y = (ctypes.c_uint64 * 4)()
    rc = lib().zkg_xyzz_to_affine(w.ctypes.data_as(u32p), x, y)
    if rc < 0:
        check(-rc)
    return None if rc == 0 else (tuple(x), tuple(y))


def xyzz_to_affine_g2(words):
    """xyzz_to_affine_g2 (src/msm.rs:356-373): 64 words -> ((x.a, x.b), (y.a, y.b)), each a
    [u64;4], or None for infinity."""
    w = as_words(words)
    assert w.size >= 64
    x = (ctypes.c_uint64 * 8)()
    y = (ctypes.c_uint64 * 8)()
    rc = lib().zkg_xyzz_to_affine_g2(w.ctypes.data_as(u32p), x, y)
    if rc < 0:
        check(-rc)
    if rc == 0:
        return None
    return ((tuple(x[0:4]), tuple(x[4:8])), (tuple(y[0:4]), tuple(y[4:8])))


def affine_words(coords, group: Group = Group.G1) -> np.ndarray:
    """The affine reading of xyzz_to_affine(_g2) back in the memory format (8 LE words per
    coordinate; zeros for infinity), as the golden vectors store results."""
    n = 16 if group == Group.G1 else 32
    out = np.zeros(n, dtype=np.uint32)
    if coords is None:
        return out
    limbs = []
    if group == Group.G1:
        limbs = [coords[0], coords[1]]
    else:
        limbs = [coords[0][0], coords[0][1], coords[1][0], coords[1][1]]
    for i, l in enumerate(limbs):
        for j, v in enumerate(l):
            out[8 * i + 2 * j] = v & 0xFFFFFFFF
            out[8 * i + 2 * j + 1] = v >> 32
    return out
