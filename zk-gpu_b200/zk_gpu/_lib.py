"""ctypes binding of libzkg.so (include/zkg.h). The library is built in-tree by
`make -C zk-gpu_b200`; importing this package without it fails loudly (there is no CPU
fallback)."""
from __future__ import annotations

import ctypes
import os

_PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.environ.get("ZKG_LIB", os.path.join(_PKG_ROOT, "libzkg.so"))

u32p = ctypes.POINTER(ctypes.c_uint32)
u64p = ctypes.POINTER(ctypes.c_uint64)
vp = ctypes.c_void_p


class StageTime(ctypes.Structure):
    _fields_ = [("stage", ctypes.c_char * 32), ("ms", ctypes.c_double)]


class MsmTuning(ctypes.Structure):
    _fields_ = [("c", ctypes.c_uint32), ("item_points", ctypes.c_uint32), ("variant", ctypes.c_int),
                ("glv", ctypes.c_int), ("ms", ctypes.c_double)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_int), ("plain", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_size_t),
                ("coset_g", ctypes.c_uint32 * 8)]


class ProofRequest(ctypes.Structure):
    _fields_ = [("log_m", ctypes.c_uint32), ("g1_scalars", ctypes.c_void_p * 3), ("g1_count", ctypes.c_size_t * 3),
                ("g2_scalars", ctypes.c_void_p), ("polys", ctypes.c_void_p * 3), ("out_points", ctypes.c_void_p),
                ("out_h", ctypes.c_void_p)]


class RequestTimes(ctypes.Structure):
    _fields_ = [("queued_ms", ctypes.c_double), ("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("slots", ctypes.c_uint64),
                ("slots_created", ctypes.c_uint64), ("slots_evicted", ctypes.c_uint64),
                ("bytes_used", ctypes.c_size_t), ("budget", ctypes.c_size_t), ("build_ms", ctypes.c_double)]


# name -> (restype, argtypes); every symbol declared in include/zkg.h
SIGNATURES = {
    "zkg_last_error": (ctypes.c_char_p, []),
    "zkg_ctx_new": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp)]),
    "zkg_ctx_free": (None, [vp]),
    "zkg_ctx_sync": (ctypes.c_int, [vp]),
    "zkg_ctx_device_name": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_size_t]),
    "zkg_buf_new": (ctypes.c_int, [vp, u32p, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_buf_zeroed": (ctypes.c_int, [vp, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_buf_write": (ctypes.c_int, [vp, vp, ctypes.c_size_t, u32p, ctypes.c_size_t]),
    "zkg_buf_read": (ctypes.c_int, [vp, vp, u32p, ctypes.c_size_t]),
    "zkg_buf_write_async": (ctypes.c_int, [vp, vp, ctypes.c_size_t, u32p, ctypes.c_size_t]),
    "zkg_buf_read_async": (ctypes.c_int, [vp, vp, u32p, ctypes.c_size_t]),
    "zkg_buf_words": (ctypes.c_size_t, [vp]),
    "zkg_buf_device_ptr": (vp, [vp]),
    "zkg_buf_free": (None, [vp]),
    "zkg_msm_default_window": (ctypes.c_uint32, [ctypes.c_size_t]),
    "zkg_msm_upload_bases": (ctypes.c_int, [vp, u32p, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_msm_upload_bases_montgomery_256": (ctypes.c_int, [vp, u32p, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_msm_new": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32,
                                   ctypes.POINTER(vp)]),
    "zkg_msm_free": (None, [vp]),
    "zkg_msm_group": (ctypes.c_int, [vp]),
    "zkg_msm_set_variant": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_set_sort": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_set_sort_form": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_fixed_base_table": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_size_t, ctypes.c_uint32,
                                                ctypes.POINTER(vp)]),
    "zkg_msm_set_fixed_base": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_set_glv": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_set_chunk": (ctypes.c_int, [vp, ctypes.c_size_t]),
    "zkg_msm_passes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "zkg_msm_windows": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_int)]),
    "zkg_xyzz_add_host": (ctypes.c_int, [ctypes.c_int, u32p, u32p, u32p]),
    "zkg_quotient": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_uint32, u32p]),
    "zkg_zkey_parse": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_zkey_free": (None, [vp]),
    "zkg_zkey_info": (ctypes.c_int, [vp, ctypes.c_void_p]),
    "zkg_zkey_points": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                       ctypes.POINTER(ctypes.c_int)]),
    "zkg_zkey_upload": (ctypes.c_int, [vp, vp, ctypes.c_uint32, ctypes.POINTER(vp)]),
    "zkg_ntt_forward_quotient": (ctypes.c_int, [vp, vp, vp, vp, u32p]),
    "zkg_msm_params": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_int)]),
    "zkg_msm_run": (ctypes.c_int, [vp, vp, vp, ctypes.POINTER(vp)]),
    "zkg_msm_profile": (ctypes.c_int, [vp, vp, vp, ctypes.POINTER(StageTime), ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_size_t)]),
    "zkg_xyzz_to_affine": (ctypes.c_int, [u32p, u64p, u64p]),
    "zkg_xyzz_to_affine_g2": (ctypes.c_int, [u32p, u64p, u64p]),
    "zkg_ntt_new": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.POINTER(vp)]),
    "zkg_ntt_free": (None, [vp]),
    "zkg_ntt_log_n": (ctypes.c_uint32, [vp]),
    "zkg_ntt_forward": (ctypes.c_int, [vp, vp]),
    "zkg_ntt_inverse": (ctypes.c_int, [vp, vp]),
    "zkg_coset_new": (ctypes.c_int, [vp, ctypes.c_uint32, u32p, ctypes.POINTER(vp)]),
    "zkg_coset_free": (None, [vp]),
    "zkg_coset_shift": (ctypes.c_int, [vp, vp]),
    "zkg_ntt_inverse_coset": (ctypes.c_int, [vp, vp, vp]),
    "zkg_batch_new": (ctypes.c_int, [vp, ctypes.POINTER(vp)]),
    "zkg_batch_free": (None, [vp]),
    "zkg_batch_add_msm": (ctypes.c_int, [vp, vp, vp, vp, vp, ctypes.c_int]),
    "zkg_batch_add_ntt": (ctypes.c_int, [vp, vp, vp, ctypes.c_int, ctypes.c_int]),
    "zkg_batch_add_coset": (ctypes.c_int, [vp, vp, vp, ctypes.c_int]),
    "zkg_batch_capture": (ctypes.c_int, [vp]),
    "zkg_batch_launch": (ctypes.c_int, [vp]),
    "zkg_batch_run_streams": (ctypes.c_int, [vp]),
    "zkg_batch_kernels": (ctypes.c_size_t, [vp]),
    "zkg_server_new": (ctypes.c_int, [vp, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]),
    "zkg_server_free": (None, [vp]),
    "zkg_server_add_key": (ctypes.c_int, [vp, ctypes.c_size_t, vp, vp]),
    "zkg_server_submit": (ctypes.c_int, [vp, ctypes.POINTER(ProofRequest), ctypes.POINTER(ctypes.c_uint64)]),
    "zkg_server_wait": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(RequestTimes)]),
    "zkg_server_stats": (ctypes.c_int, [vp, ctypes.POINTER(ServerStats)]),
    "zkg_server_reserve": (ctypes.c_int, [vp, ctypes.c_uint32, ctypes.c_uint32]),
    "zkg_tune_msm": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_size_t, vp, vp, ctypes.c_int,
                                    ctypes.POINTER(MsmTuning), ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "zkg_ntt_set_variant": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_ntt_set_max_stages": (ctypes.c_int, [vp, ctypes.c_uint32]),
    "zkg_ntt_params": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_uint32),
                                      ctypes.POINTER(ctypes.c_uint32)]),
    "zkg_tune_ntt": (ctypes.c_int, [vp, ctypes.c_uint32, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_double)]),
    "zkg_ntt_noalloc": (ctypes.c_int, [ctypes.c_uint32, ctypes.c_int, vp, vp]),
    "zkg_ctx_stream": (vp, [vp]),
    "zkg_launch_count": (ctypes.c_uint64, []),
    "zkg_host_alloc": (ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(vp)]),
    "zkg_host_free": (None, [vp]),
    "zkg_msm_set_timing": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_msm_stage_times": (ctypes.c_int, [vp, ctypes.POINTER(StageTime), ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "zkg_msm_last_entries": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_uint64)]),
    "zkg_ntt_set_timing": (ctypes.c_int, [vp, ctypes.c_int]),
    "zkg_ntt_pass_times": (ctypes.c_int, [vp, ctypes.POINTER(StageTime), ctypes.c_size_t,
                                          ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "zkg_bench_integer_pipe": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "zkg_test_point_ops": (ctypes.c_int, [vp, ctypes.c_int, u32p, ctypes.c_size_t, u32p]),
    "zkg_test_glv_split": (ctypes.c_int, [vp, u32p, ctypes.c_size_t, u32p]),
    "zkg_generator_multiples": (ctypes.c_int, [vp, ctypes.c_int, vp, ctypes.c_size_t, ctypes.c_int, vp]),
}

_lib = None


def lib():
    """The loaded library (raises OSError when libzkg.so has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C zk-gpu_b200` "
                          "(the CUDA library is required; there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class ZkGpuError(RuntimeError):
    """A failed call; `code` is the zkg_status value, the message is the library's (the same
    text as the reference's panic for argument errors)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


def check(rc: int) -> None:
    if rc != 0:
        msg = lib().zkg_last_error()
        raise ZkGpuError(rc, msg.decode() if msg else f"zkg error {rc}")
