"""GPU results against the reference's golden vectors (tests/golden.rs:15-56): ffjavascript
outputs, independent of arkworks and of this library."""
import numpy as np
import pytest

from common import golden_msm_cases, golden_ntt_cases
from zk_gpu import Msm, Ntt, xyzz_to_affine
from zk_gpu.msm import affine_words

pytestmark = pytest.mark.gpu


def test_ntt_matches_ffjavascript(gpu):
    for log_n, inverse, inp, out in golden_ntt_cases():
        ntt = Ntt(gpu, log_n)
        buf = gpu.buffer(inp)
        (ntt.inverse if inverse else ntt.forward)(gpu, buf)
        got = gpu.read(buf, inp.size)
        assert np.array_equal(got, out), f"NTT (log_n = {log_n}, inverse = {inverse}) differs from ffjavascript"


def test_msm_matches_ffjavascript(gpu):
    for name, bases, scalars, result in golden_msm_cases():
        n = scalars.size // 8
        base_buf = Msm.upload_bases(gpu, bases)
        scalar_buf = gpu.buffer(scalars)
        # Library defaults, a small window with tiny work items, and a large window.
        for plan in [None, (9, 7), (12, 1024)]:
            msm = Msm(gpu, n, Msm.default_window(n)) if plan is None else Msm.with_item_points(gpu, n, *plan)
            out = msm.run(gpu, base_buf, scalar_buf)
            got = affine_words(xyzz_to_affine(gpu.read(out, 32)))
            assert np.array_equal(got, result), f"MSM '{name}' (n = {n}, plan = {plan}) differs from ffjavascript"
