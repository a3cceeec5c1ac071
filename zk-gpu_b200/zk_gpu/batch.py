"""Batched execution over zkg_batch: MSMs, NTTs and coset shifts of uneven sizes captured into
one CUDA graph (lanes are independent branches) and replayed with one launch."""
from __future__ import annotations

import ctypes

from ._lib import check, lib, vp
from .gpu import Buffer, Gpu
from .msm import Msm
from .ntt import CosetShift, Ntt


class Batch:
    def __init__(self, gpu: Gpu):
        h = vp()
        check(lib().zkg_batch_new(gpu.handle, ctypes.byref(h)))
        self._h = h.value
        self._gpu = gpu
        self._keep = []  # plans and buffers must outlive the batch

    def add_msm(self, msm: Msm, bases: Buffer, scalars: Buffer, result: Buffer | None = None, lane: int = 0):
        check(lib().zkg_batch_add_msm(self._h, msm._h, bases.handle, scalars.handle,
                                      result.handle if result is not None else None, lane))
        self._keep += [msm, bases, scalars, result]

    def add_ntt(self, ntt: Ntt, data: Buffer, inverse: bool = False, lane: int = 0):
        check(lib().zkg_batch_add_ntt(self._h, ntt.handle, data.handle, int(inverse), lane))
        self._keep += [ntt, data]

    def add_coset(self, coset: CosetShift, data: Buffer, lane: int = 0):
        check(lib().zkg_batch_add_coset(self._h, coset.handle, data.handle, lane))
        self._keep += [coset, data]

    def capture(self):
        check(lib().zkg_batch_capture(self._h))

    def launch(self):
        """One graph launch for every recorded operation (captures first if needed)."""
        check(lib().zkg_batch_launch(self._h))

    def run_streams(self):
        """The same operations without a graph, one stream per lane."""
        check(lib().zkg_batch_run_streams(self._h))

    def kernels(self) -> int:
        return lib().zkg_batch_kernels(self._h)

    def close(self):
        if self._h:
            lib().zkg_batch_free(self._h)
        self._h = None
        self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
