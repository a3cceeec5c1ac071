"""snarkjs Groth16 proving keys (.zkey) over zkg_zkey: parse a file image on the host, then
upload its point sections as resident MSM bases (the Montgomery-2^256 form that
Msm::upload_bases_montgomery_256 takes as it is, src/msm.rs:190-197)."""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import check, lib, vp
from .gpu import Buffer, Gpu
from .group import Group

IC, A, B1, B2, C, H = 3, 5, 6, 7, 8, 9


class ZkeyHeader(ctypes.Structure):
    _fields_ = [("protocol", ctypes.c_uint32), ("n_vars", ctypes.c_uint32), ("n_public", ctypes.c_uint32),
                ("domain_size", ctypes.c_uint32)]


class Zkey:
    def __init__(self, data: bytes):
        h = vp()
        buf = ctypes.create_string_buffer(bytes(data), len(data))
        check(lib().zkg_zkey_parse(buf, len(data), ctypes.byref(h)))
        self._h = h.value

    @classmethod
    def open(cls, path: str) -> "Zkey":
        with open(path, "rb") as f:
            return cls(f.read())

    def header(self) -> dict:
        hd = ZkeyHeader()
        check(lib().zkg_zkey_info(self._h, ctypes.byref(hd)))
        return {"protocol": hd.protocol, "n_vars": hd.n_vars, "n_public": hd.n_public,
                "domain_size": hd.domain_size}

    def points(self, section: int) -> tuple[np.ndarray, Group]:
        """The section's words as the file holds them (16 / 32 words per G1 / G2 point)."""
        w = ctypes.POINTER(ctypes.c_uint32)()
        pts, grp = ctypes.c_size_t(), ctypes.c_int()
        check(lib().zkg_zkey_points(self._h, section, ctypes.byref(w), ctypes.byref(pts), ctypes.byref(grp)))
        group = Group.G1 if grp.value == 1 else Group.G2
        words = pts.value * group.affine_words()
        arr = np.ctypeslib.as_array(w, shape=(words,)).copy() if words else np.zeros(0, dtype=np.uint32)
        return arr, group

    def upload(self, gpu: Gpu, section: int) -> Buffer:
        h = vp()
        check(lib().zkg_zkey_upload(gpu.handle, self._h, section, ctypes.byref(h)))
        return Buffer(gpu, h.value)

    def close(self) -> None:
        if self._h:
            lib().zkg_zkey_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
