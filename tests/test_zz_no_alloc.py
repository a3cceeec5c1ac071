"""zkg_ntt_noalloc, the NTT entry point that allocates no device memory (for callers that may
not call cudaMalloc: a device-memory budget owned by another allocator, or a pipeline where
allocation is not allowed). It must give exactly what the plan-based zkg_ntt_forward /
zkg_ntt_inverse give, call after call, although every call reuses one static scratch array.

Collected last on purpose (file name), so a failure here comes after every other test ran."""
import ctypes

import numpy as np
import pytest

from common import random_fr
from zk_gpu import Ntt, ZkGpuError, lib
from zk_gpu._lib import check

pytestmark = pytest.mark.gpu


def noalloc(gpu, buf, log_n, inverse):
    stream = lib().zkg_ctx_stream(gpu.handle)
    check(lib().zkg_ntt_noalloc(log_n, int(inverse), buf.device_ptr(), stream))


def plan_result(gpu, x, log_n, inverse):
    buf = gpu.buffer(x)
    ntt = Ntt(gpu, log_n)
    (ntt.inverse if inverse else ntt.forward)(gpu, buf)
    return gpu.read(buf, x.size)


def test_matches_the_plan_entry_points_call_after_call(gpu):
    # Two calls in a row on the largest size, then a smaller size and back: the shared scratch
    # keeps each call's contents, which must never leak into the next result.
    # log_n 10 and 11 take the one-pass branch (the tile is the whole transform and the scratch
    # array holds only the twiddles).
    cases = [(16, False, 1), (16, True, 2), (12, True, 3), (16, False, 4), (10, False, 6), (10, True, 7),
             (11, False, 8), (11, True, 9), (16, True, 10)]
    for log_n, inverse, seed in cases:
        x = random_fr(seed, 1 << log_n)
        buf = gpu.buffer(x)
        noalloc(gpu, buf, log_n, inverse)
        got = gpu.read(buf, x.size)
        assert np.array_equal(got, plan_result(gpu, x, log_n, inverse)), (log_n, inverse)


@pytest.mark.parametrize("log_n", [10, 11, 14])
def test_round_trip(gpu, log_n):
    x = random_fr(5 + log_n, 1 << log_n)
    buf = gpu.buffer(x)
    noalloc(gpu, buf, log_n, False)
    noalloc(gpu, buf, log_n, True)
    assert np.array_equal(gpu.read(buf, x.size), x)


def test_sizes_beyond_the_scratch_are_rejected(gpu):
    buf = gpu.buffer(np.zeros(8 << 17, dtype=np.uint32))
    with pytest.raises(ZkGpuError, match=r"log_n must be in 10..=16 for zkg_ntt_noalloc, got 17"):
        noalloc(gpu, buf, 17, False)
    with pytest.raises(ZkGpuError, match="data is NULL"):
        check(lib().zkg_ntt_noalloc(12, 0, None, lib().zkg_ctx_stream(gpu.handle)))
    assert ctypes.sizeof(ctypes.c_void_p) == 8
