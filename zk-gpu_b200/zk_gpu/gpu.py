"""gpu::Gpu and its buffers (src/gpu.rs:6-199) over zkg_ctx / zkg_buf."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib, u32p, vp


def as_words(data) -> np.ndarray:
    """u32 words as a C-contiguous numpy array (lists, arrays and bytes accepted)."""
    if isinstance(data, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(data), dtype=np.uint32)
    return np.ascontiguousarray(data, dtype=np.uint32)


class Buffer:
    """A device buffer of u32 words (wgpu::Buffer with STORAGE usage, src/gpu.rs:57-69)."""

    def __init__(self, gpu: "Gpu", handle: int, owned: bool = True):
        self.gpu = gpu
        self._h = handle
        self._owned = owned

    @property
    def handle(self) -> int:
        return self._h

    def words(self) -> int:
        return lib().zkg_buf_words(self._h)

    def size(self) -> int:
        """Size in bytes (wgpu::Buffer::size)."""
        return 4 * self.words()

    def device_ptr(self) -> int:
        return lib().zkg_buf_device_ptr(self._h) or 0

    def write(self, data, offset_words: int = 0) -> None:
        w = as_words(data)
        check(lib().zkg_buf_write(self.gpu.handle, self._h, offset_words, w.ctypes.data_as(u32p), w.size))

    def write_async(self, data: np.ndarray, offset_words: int = 0) -> None:
        """Queued write (zkg_buf_write_async): `data` (u32 words, ideally page-locked) must stay
        unchanged until Gpu.wait(); the Gpu keeps a reference until then."""
        if data.dtype != np.uint32 or not data.flags["C_CONTIGUOUS"]:
            raise ValueError("write_async needs a contiguous uint32 array")
        check(lib().zkg_buf_write_async(self.gpu.handle, self._h, offset_words, data.ctypes.data_as(u32p), data.size))
        self.gpu._pending.append(data)

    def free(self) -> None:
        if self._h and self._owned:
            lib().zkg_buf_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Gpu:
    """One CUDA device with one ordered stream (gpu::Gpu, src/gpu.rs:6-55)."""

    def __init__(self, device: int = 0):
        h = vp()
        check(lib().zkg_ctx_new(device, ctypes.byref(h)))
        self._h = h.value
        self._pending = []  # host arrays of queued asynchronous copies, held until wait()

    @classmethod
    def new(cls, device: int = 0) -> "Gpu":
        return cls(device)

    @property
    def handle(self) -> int:
        return self._h

    @property
    def adapter_name(self) -> str:
        out = ctypes.create_string_buffer(256)
        check(lib().zkg_ctx_device_name(self._h, out, 256))
        return out.value.decode()

    def buffer(self, data) -> Buffer:
        """Gpu::buffer: storage buffer initialised with `data` (u32 words)."""
        w = as_words(data)
        h = vp()
        check(lib().zkg_buf_new(self._h, w.ctypes.data_as(u32p), w.size, ctypes.byref(h)))
        return Buffer(self, h.value)

    def empty_buffer(self, words: int) -> Buffer:
        """Gpu::empty_buffer: zero-filled buffer of `words` u32s."""
        h = vp()
        check(lib().zkg_buf_zeroed(self._h, words, ctypes.byref(h)))
        return Buffer(self, h.value)

    def read(self, buffer: Buffer, words: int) -> np.ndarray:
        """Gpu::read: blocking read of the first `words` words."""
        out = np.empty(words, dtype=np.uint32)
        check(lib().zkg_buf_read(self._h, buffer.handle, out.ctypes.data_as(u32p), words))
        return out

    def read_async(self, buffer: Buffer, out: np.ndarray) -> None:
        """Queued read (zkg_buf_read_async) of out.size words into `out` (a contiguous uint32
        array, ideally page-locked), valid after wait()."""
        if out.dtype != np.uint32 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("read_async needs a contiguous uint32 array")
        check(lib().zkg_buf_read_async(self._h, buffer.handle, out.ctypes.data_as(u32p), out.size))
        self._pending.append(out)

    def wait(self) -> None:
        """Gpu::wait: block until all queued work (kernels and asynchronous copies) has finished."""
        check(lib().zkg_ctx_sync(self._h))
        self._pending.clear()

    def close(self) -> None:
        if self._h:
            lib().zkg_ctx_free(self._h)
        self._h = None
