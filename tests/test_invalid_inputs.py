"""Wrong sizes and parameters fail loudly with the reference's messages
(tests/invalid_inputs.rs:8-59); oversized buffers are accepted."""
import numpy as np
import pytest

from zk_gpu import Msm, Ntt, ZkGpuError

pytestmark = pytest.mark.gpu
N = 4096


def test_msm_with_no_points(gpu):
    with pytest.raises(ZkGpuError, match="at least one point"):
        Msm(gpu, 0, 10)


def test_msm_window_out_of_range(gpu):
    with pytest.raises(ZkGpuError, match=r"window size c must be in 9..=20"):
        Msm(gpu, N, 8)
    with pytest.raises(ZkGpuError, match=r"window size c must be in 9..=20, got 21"):
        Msm(gpu, N, 21)


def test_msm_scalars_too_small(gpu):
    bases = Msm.upload_bases(gpu, np.zeros(16 * N, dtype=np.uint32))
    scalars = gpu.buffer(np.ones(4 * N, dtype=np.uint32))  # half of what 4096 scalars need
    with pytest.raises(ZkGpuError, match="scalars buffer holds"):
        Msm(gpu, N, 10).run(gpu, bases, scalars)


def test_msm_bases_too_small(gpu):
    bases = Msm.upload_bases(gpu, np.zeros(8 * N, dtype=np.uint32))  # half of what 4096 points need
    scalars = gpu.buffer(np.ones(8 * N, dtype=np.uint32))
    with pytest.raises(ZkGpuError, match="bases buffer holds"):
        Msm(gpu, N, 10).run(gpu, bases, scalars)


def test_ntt_size_out_of_range(gpu):
    with pytest.raises(ZkGpuError, match=r"log_n must be in 10..=27"):
        Ntt(gpu, 9)
    with pytest.raises(ZkGpuError, match=r"log_n must be in 10..=27"):
        Ntt(gpu, 28)


def test_ntt_data_too_small(gpu):
    data = gpu.buffer(np.ones(8 << 11, dtype=np.uint32))  # half of a 2^12 transform
    with pytest.raises(ZkGpuError, match="data buffer holds"):
        Ntt(gpu, 12).forward(gpu, data)


def test_buffers_larger_than_needed_are_accepted(gpu):
    data = gpu.buffer(np.ones(8 << 13, dtype=np.uint32))  # room for 2^13, transform of 2^12
    ntt = Ntt(gpu, 12)
    ntt.forward(gpu, data)
    ntt.inverse(gpu, data)
    back = gpu.read(data, 8 << 13)
    assert np.array_equal(back, np.ones(8 << 13, dtype=np.uint32))


def test_tuning_knobs_reject_out_of_range_values(gpu):
    """The plan knobs of this library (no reference counterpart) reject unknown forms."""
    from zk_gpu import Group
    g1 = Msm(gpu, 1 << 10, 10)
    with pytest.raises(ZkGpuError, match="accumulation variant must be 0..6"):
        g1.set_variant(7)
    with pytest.raises(ZkGpuError, match="sort aggregation mode must be 0..3"):
        g1.set_sort(4)
    g2 = Msm.for_group(gpu, Group.G2, 1 << 10, 10)
    with pytest.raises(ZkGpuError, match="accumulation variant must be 0..6"):
        g2.set_variant(-1)
    assert g2.params()["variant"] == 2 and g1.params()["variant"] == 4  # G1: the GLV split's default form
    assert Msm(gpu, 1 << 23, 16).params()["variant"] == 4  # 2^27 entries: one product per call
    ntt = Ntt(gpu, 12)
    with pytest.raises(ZkGpuError, match="NTT variant must be 0..4"):
        ntt.set_variant(5)
    with pytest.raises(ZkGpuError, match=r"max_stages must be in 6..=10"):
        ntt.set_max_stages(11)
    ntt.set_variant(0)
    with pytest.raises(ZkGpuError, match=r"max_stages must be in 6..=11"):
        ntt.set_max_stages(12)
