"""Queued buffer copies (zkg_buf_write_async / zkg_buf_read_async) keep the order of the work
around them: a write waits for queued work that still uses the buffer, later work waits for the
write, and a read sees the data of the work queued before it."""
import numpy as np
import pytest

from common import msm_ref, random_fr, random_points
from oracle import cpu
from zk_gpu import Batch, Msm, Ntt, ZkGpuError, xyzz_to_affine
from zk_gpu.msm import affine_words
from zk_gpu.serving import PinnedWords

pytestmark = pytest.mark.gpu


def pinned(values: np.ndarray) -> PinnedWords:
    p = PinnedWords(values.size)
    p.array[:] = values
    return p


def test_round_trip_through_page_locked_memory(gpu):
    x = random_fr(1, 1 << 16)
    src, dst = pinned(x), PinnedWords(x.size)
    buf = gpu.empty_buffer(x.size)
    buf.write_async(src.array)
    gpu.read_async(buf, dst.array)
    gpu.wait()
    assert np.array_equal(dst.array, x)
    # pageable arrays work too (the copy just does not overlap)
    y = random_fr(2, 1000)
    buf.write_async(y, offset_words=8)
    out = np.zeros(1000, dtype=np.uint32)
    gpu.read_async(buf, out)
    gpu.wait()
    assert np.array_equal(out[8:], y[:992])


def test_write_waits_for_queued_readers_of_the_buffer(gpu):
    """Scalars overwritten right after an MSM that reads them was queued: the MSM sees the old
    values, the next MSM the new ones."""
    n = 1 << 15
    bases = random_points("G1", 3, n)
    s_old, s_new = random_fr(4, n), random_fr(5, n)
    base_buf, sbuf = Msm.upload_bases(gpu, bases), gpu.buffer(s_old)
    msm_a, msm_b = Msm(gpu, n, Msm.default_window(n)), Msm(gpu, n, Msm.default_window(n))
    res_a, res_b = PinnedWords(32), PinnedWords(32)
    new = pinned(s_new)
    ra = msm_a.run(gpu, base_buf, sbuf)
    sbuf.write_async(new.array)
    rb = msm_b.run(gpu, base_buf, sbuf)
    gpu.read_async(ra, res_a.array)
    gpu.read_async(rb, res_b.array)
    gpu.wait()
    assert np.array_equal(affine_words(xyzz_to_affine(res_a.array)), msm_ref("G1", bases, s_old))
    assert np.array_equal(affine_words(xyzz_to_affine(res_b.array)), msm_ref("G1", bases, s_new))


def test_reads_between_transforms_of_one_buffer(gpu):
    """forward, read, inverse, read on one buffer: each read sees its transform's output."""
    log_n = 16
    x = random_fr(6, 1 << log_n)
    ntt = Ntt(gpu, log_n)
    buf = gpu.empty_buffer(x.size)
    src, fwd, back = pinned(x), PinnedWords(x.size), PinnedWords(x.size)
    for _ in range(2):  # the second round reuses the page-locked arrays
        buf.write_async(src.array)
        ntt.forward(gpu, buf)
        gpu.read_async(buf, fwd.array)
        ntt.inverse(gpu, buf)
        gpu.read_async(buf, back.array)
        gpu.wait()
        assert np.array_equal(fwd.array, cpu.ntt(x))
        assert np.array_equal(back.array, x)


def test_write_waits_for_a_queued_batch(gpu):
    n = 1 << 12
    bases = random_points("G1", 7, n)
    s_old, s_new = random_fr(8, n), random_fr(9, n)
    base_buf, sbuf = Msm.upload_bases(gpu, bases), gpu.buffer(s_old)
    out = gpu.empty_buffer(32)
    batch = Batch(gpu)
    batch.add_msm(Msm(gpu, n, Msm.default_window(n)), base_buf, sbuf, out, lane=0)
    batch.launch()
    new = pinned(s_new)  # the page-locked source stays alive until the copy has run
    sbuf.write_async(new.array)
    res = PinnedWords(32)
    gpu.read_async(out, res.array)
    gpu.wait()
    assert np.array_equal(affine_words(xyzz_to_affine(res.array)), msm_ref("G1", bases, s_old))
    batch.close()


def test_async_copies_check_sizes(gpu):
    buf = gpu.empty_buffer(16)
    with pytest.raises(ZkGpuError, match="overruns a buffer of 16 words"):
        buf.write_async(np.zeros(17, dtype=np.uint32))
    with pytest.raises(ZkGpuError, match="from a buffer of 16"):
        gpu.read_async(buf, np.zeros(17, dtype=np.uint32))


def test_next_upload_waits_for_a_queued_read_of_the_buffer(gpu):
    """A read queued on the read-back stream, then a write of new data into the same buffer on
    the upload stream: the read still returns the old contents."""
    x, y = random_fr(10, 1 << 16), random_fr(11, 1 << 16)
    buf = gpu.buffer(x)
    ntt = Ntt(gpu, 16)
    ntt.forward(gpu, buf)
    out = PinnedWords(x.size)
    gpu.read_async(buf, out.array)
    new = pinned(y)
    buf.write_async(new.array)
    back = PinnedWords(x.size)
    gpu.read_async(buf, back.array)
    gpu.wait()
    assert np.array_equal(out.array, cpu.ntt(x))
    assert np.array_equal(back.array, y)


def test_read_back_overlaps_later_work_but_not_later_writers(gpu):
    """A read of an NTT output does not hold back an MSM queued after it, but the next transform
    of the same buffer (which overwrites it) waits for the read; the MSM plan's result is read
    before the next run of that plan overwrites it."""
    log_n, n = 16, 1 << 14
    x, y = random_fr(20, 1 << log_n), random_fr(21, 1 << log_n)
    bases = random_points("G1", 22, n)
    s1, s2 = random_fr(23, n), random_fr(24, n)
    base_buf, sbuf1, sbuf2 = Msm.upload_bases(gpu, bases), gpu.buffer(s1), gpu.buffer(s2)
    ntt = Ntt(gpu, log_n)
    msm = Msm(gpu, n, Msm.default_window(n))
    data = gpu.buffer(x)
    fwd_x, fwd_y = PinnedWords(x.size), PinnedWords(x.size)
    res1, res2 = PinnedWords(32), PinnedWords(32)
    new = pinned(y)
    for _ in range(2):
        ntt.forward(gpu, data)
        gpu.read_async(data, fwd_x.array)    # read of the first transform's output
        r = msm.run(gpu, base_buf, sbuf1)    # independent work: runs alongside the read
        gpu.read_async(r, res1.array)
        r = msm.run(gpu, base_buf, sbuf2)    # overwrites the plan's result: waits for that read
        gpu.read_async(r, res2.array)
        data.write_async(new.array)          # overwrites data: waits for the first read
        ntt.forward(gpu, data)
        gpu.read_async(data, fwd_y.array)
        ntt.inverse(gpu, data)               # overwrites data: waits for the second read
        gpu.wait()
        assert np.array_equal(fwd_x.array, cpu.ntt(x))
        assert np.array_equal(fwd_y.array, cpu.ntt(y))
        assert np.array_equal(gpu.read(data, y.size), y)
        assert np.array_equal(affine_words(xyzz_to_affine(res1.array)), msm_ref("G1", bases, s1))
        assert np.array_equal(affine_words(xyzz_to_affine(res2.array)), msm_ref("G1", bases, s2))
        data.write(x)


def test_synchronous_write_then_queued_read(gpu):
    """A blocking write from pageable memory followed by a queued read returns the new words."""
    buf = gpu.buffer(random_fr(25, 4096))
    y = random_fr(26, 4096)
    out = PinnedWords(y.size)
    ntt = Ntt(gpu, 12)
    ntt.forward(gpu, buf)          # an older recorded use of the buffer
    buf.write(y)
    gpu.read_async(buf, out.array)
    gpu.wait()
    assert np.array_equal(out.array, y)
