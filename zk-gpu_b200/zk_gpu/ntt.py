"""ntt::Ntt (src/ntt.rs:14-50) over zkg_ntt."""
from __future__ import annotations

import ctypes

from ._lib import check, lib, vp
from .gpu import Buffer, Gpu


class Ntt:
    """Plan for in-place transforms of 2^log_n Fr elements (10 <= log_n <= 27), natural order
    in and out; buffers hold 8 plain u32 words per element."""

    def __init__(self, gpu: Gpu, log_n: int):
        h = vp()
        check(lib().zkg_ntt_new(gpu.handle, log_n, ctypes.byref(h)))
        self._h = h.value
        self._gpu = gpu

    @classmethod
    def new(cls, gpu: Gpu, log_n: int) -> "Ntt":
        return cls(gpu, log_n)

    @property
    def log_n(self) -> int:
        return lib().zkg_ntt_log_n(self._h)

    @property
    def handle(self) -> int:
        return self._h

    def forward(self, gpu: Gpu, data: Buffer) -> None:
        """In-place forward transform (Radix2EvaluationDomain::fft)."""
        check(lib().zkg_ntt_forward(self._h, data.handle))

    def inverse(self, gpu: Gpu, data: Buffer) -> None:
        """In-place inverse transform, including the 1/n factor."""
        check(lib().zkg_ntt_inverse(self._h, data.handle))

    def inverse_coset(self, gpu: Gpu, data: Buffer, coset: "CosetShift") -> None:
        """inverse() then coset.shift() in one call: the shift runs in the inverse's last pass."""
        check(lib().zkg_ntt_inverse_coset(self._h, data.handle, coset.handle))

    def forward_quotient(self, gpu: Gpu, data: Buffer, a: Buffer, b: Buffer, g: int) -> None:
        """forward() of data (c on the coset g*H), then data <- (a * b - data) / (g^N - 1), the
        quotient running in the transform's last pass."""
        check(lib().zkg_ntt_forward_quotient(self._h, data.handle, a.handle, b.handle, _fr_words(g)))

    def set_variant(self, variant: int) -> None:
        """Butterfly form: 0 = 32-bit integer products, 1 = double-precision limbs with twiddles
        read from a table of powers, 2 = double-precision limbs with each stage's twiddles staged
        into shared memory, 3 = form 2 with two butterflies per thread step."""
        check(lib().zkg_ntt_set_variant(self._h, variant))

    def set_max_stages(self, max_stages: int) -> None:
        check(lib().zkg_ntt_set_max_stages(self._h, max_stages))

    def params(self) -> dict:
        v, ms, p = ctypes.c_int(), ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().zkg_ntt_params(self._h, ctypes.byref(v), ctypes.byref(ms), ctypes.byref(p)))
        return {"variant": v.value, "max_stages": ms.value, "passes": p.value}

    def close(self) -> None:
        if self._h:
            lib().zkg_ntt_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _fr_words(v: int):
    import numpy as np

    from ._lib import u32p
    words = np.array([(v >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)
    _fr_words.keep = words  # alive for the call
    return words.ctypes.data_as(u32p)


def quotient(gpu: Gpu, a: Buffer, b: Buffer, c: Buffer, log_n: int, g: int) -> None:
    """a <- (a * b - c) / (g^N - 1), N = 2^log_n: the pointwise step of a Groth16 witness map on
    the coset g*H (plain Fr words, natural order)."""
    check(lib().zkg_quotient(gpu.handle, a.handle, b.handle, c.handle, log_n, _fr_words(g)))


class CosetShift:
    """x_i <- x_i * g^i over the first 2^log_n elements, g a fixed Fr element (int < r)."""

    def __init__(self, gpu: Gpu, log_n: int, g: int):
        import numpy as np

        from ._lib import u32p
        words = np.array([(g >> (32 * i)) & 0xFFFFFFFF for i in range(8)], dtype=np.uint32)
        h = vp()
        check(lib().zkg_coset_new(gpu.handle, log_n, words.ctypes.data_as(u32p), ctypes.byref(h)))
        self._h = h.value

    @property
    def handle(self) -> int:
        return self._h

    def shift(self, gpu: Gpu, data: Buffer) -> None:
        check(lib().zkg_coset_shift(self._h, data.handle))

    def close(self) -> None:
        if self._h:
            lib().zkg_coset_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
