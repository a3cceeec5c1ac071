"""ctypes front end of the C oracle (oracle/zkg_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the tests, the smoke check and bench.py's CPU-baseline
leg, never by the product library. All arrays are numpy uint32 in the reference's memory
format: 8 little-endian u32 words per field element (src/host.rs:104-110), affine points as
x then y (Fq2 as a then b), infinity as all-zero words (src/msm.rs:182-183).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libzkg_oracle.so")
_lib = None

_u32p = ctypes.POINTER(ctypes.c_uint32)


def build() -> str:
    """Compiles the oracle with its Makefile (gcc); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_msm.argtypes = [ctypes.c_int, _u32p, ctypes.c_int, _u32p, ctypes.c_size_t,
                                 ctypes.c_int, ctypes.c_int, _u32p]
        L.oracle_msm.restype = ctypes.c_int
        L.oracle_generator_multiples.argtypes = [ctypes.c_int, _u32p, ctypes.c_size_t, ctypes.c_int,
                                                 ctypes.c_int, _u32p]
        L.oracle_generator_multiples.restype = ctypes.c_int
        L.oracle_fr_dot.argtypes = [_u32p, _u32p, ctypes.c_size_t, ctypes.c_int, _u32p]
        L.oracle_fr_dot.restype = None
        L.oracle_scalar_mul.argtypes = [ctypes.c_int, _u32p, _u32p, _u32p]
        L.oracle_scalar_mul.restype = None
        L.oracle_ntt.argtypes = [_u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_ntt.restype = ctypes.c_int
        L.oracle_ntt_eval.argtypes = [_u32p, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, _u32p]
        L.oracle_ntt_eval.restype = None
        L.oracle_coset_shift.argtypes = [_u32p, ctypes.c_size_t, _u32p]
        L.oracle_coset_shift.restype = None
        L.oracle_fq_to_mont256.argtypes = [_u32p, ctypes.c_size_t]
        L.oracle_fq_to_mont256.restype = None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u32p)


def threads() -> int:
    return os.cpu_count() or 1


def group_id(group: str) -> int:
    return 1 if group == "G1" else 2


def msm(group: str, bases: np.ndarray, scalars: np.ndarray, mont256: bool = False,
        c: int = 0, nthreads: int | None = None) -> np.ndarray:
    """sum_i s_i * P_i; returns plain affine words (16 G1 / 32 G2; zeros = infinity)."""
    aw = 16 if group == "G1" else 32
    bases = np.ascontiguousarray(bases, dtype=np.uint32)
    scalars = np.ascontiguousarray(scalars, dtype=np.uint32)
    n = scalars.size // 8
    assert bases.size >= n * aw
    out = np.zeros(aw, dtype=np.uint32)
    rc = lib().oracle_msm(group_id(group), _p(bases), int(mont256), _p(scalars), n, c,
                          nthreads or threads(), _p(out))
    if rc != 0:
        raise ValueError(f"oracle_msm failed ({rc})")
    return out


def generator_multiples(group: str, k: np.ndarray, mont256: bool = False,
                        nthreads: int | None = None) -> np.ndarray:
    """[k_i]G (G1 = (1,2), G2 = the standard generator) as affine words."""
    aw = 16 if group == "G1" else 32
    k = np.ascontiguousarray(k, dtype=np.uint32)
    n = k.size // 8
    out = np.zeros(n * aw, dtype=np.uint32)
    lib().oracle_generator_multiples(group_id(group), _p(k), n, nthreads or threads(), int(mont256), _p(out))
    return out


def fr_dot(a: np.ndarray, b: np.ndarray, nthreads: int | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint32)
    b = np.ascontiguousarray(b, dtype=np.uint32)
    out = np.zeros(8, dtype=np.uint32)
    lib().oracle_fr_dot(_p(a), _p(b), a.size // 8, nthreads or threads(), _p(out))
    return out


def scalar_mul(group: str, point: np.ndarray, k: np.ndarray) -> np.ndarray:
    aw = 16 if group == "G1" else 32
    point = np.ascontiguousarray(point, dtype=np.uint32)
    k = np.ascontiguousarray(k, dtype=np.uint32)
    out = np.zeros(aw, dtype=np.uint32)
    lib().oracle_scalar_mul(group_id(group), _p(point), _p(k), _p(out))
    return out


def ntt(data: np.ndarray, inverse: bool = False, nthreads: int | None = None) -> np.ndarray:
    """Returns the transform of `data` (a copy): natural order in and out."""
    out = np.array(data, dtype=np.uint32, copy=True)
    log_n = (out.size // 8).bit_length() - 1
    assert (1 << log_n) * 8 == out.size
    rc = lib().oracle_ntt(_p(out), log_n, int(inverse), nthreads or threads())
    if rc != 0:
        raise ValueError(f"oracle_ntt failed ({rc})")
    return out


def ntt_eval(data: np.ndarray, k: int, inverse: bool = False) -> np.ndarray:
    data = np.ascontiguousarray(data, dtype=np.uint32)
    log_n = (data.size // 8).bit_length() - 1
    out = np.zeros(8, dtype=np.uint32)
    lib().oracle_ntt_eval(_p(data), log_n, k, int(inverse), _p(out))
    return out


def coset_shift(data: np.ndarray, g_words: np.ndarray) -> np.ndarray:
    out = np.array(data, dtype=np.uint32, copy=True)
    g = np.ascontiguousarray(g_words, dtype=np.uint32)
    lib().oracle_coset_shift(_p(out), out.size // 8, _p(g))
    return out


def fq_to_mont256(words: np.ndarray) -> np.ndarray:
    out = np.array(words, dtype=np.uint32, copy=True)
    lib().oracle_fq_to_mont256(_p(out), out.size // 8)
    return out
