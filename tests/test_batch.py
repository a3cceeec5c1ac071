"""Batched execution (one CUDA graph, lanes as independent branches) gives exactly the oracle's
results, and the same as the operations run one call at a time."""
import numpy as np
import pytest

from common import msm_ref, random_fr, random_points
from oracle import bn254, cpu
from zk_gpu import Batch, CosetShift, Group, Msm, Ntt, ZkGpuError, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words

pytestmark = pytest.mark.gpu


def plain_msm(gpu, group, bases_buf, scalars, n):
    msm = Msm.for_group(gpu, group, n, Msm.default_window(n))
    words = gpu.read(msm.run(gpu, bases_buf, gpu.buffer(scalars)), group.xyzz_words())
    conv = xyzz_to_affine if group == Group.G1 else xyzz_to_affine_g2
    return affine_words(conv(words), group)


def test_uneven_batch_matches_single_calls(gpu):
    rnd_sizes = [(Group.G1, 1000), (Group.G1, 1 << 14), (Group.G2, 3000), (Group.G1, 1 << 17)]
    batch = Batch(gpu)
    expected, outputs = [], []
    for lane, (group, n) in enumerate(rnd_sizes):
        gname = "G1" if group == Group.G1 else "G2"
        points = random_points(gname, 500 + lane, n)
        bases = Msm.upload_bases(gpu, points)
        for rep in range(2):  # two MSMs with the same plan in one lane
            s = random_fr(600 + 10 * lane + rep, n)
            sbuf = gpu.buffer(s)
            if rep == 0:
                plan = Msm.for_group(gpu, group, n, Msm.default_window(n))
            out = gpu.empty_buffer(group.xyzz_words())
            batch.add_msm(plan, bases, sbuf, out, lane=lane)
            outputs.append((group, out))
            want = msm_ref(gname, points, s)
            assert np.array_equal(plain_msm(gpu, group, bases, s, n), want), (gname, n)
            expected.append(want)
    # an NTT chain (inverse, coset shift, forward) in its own lane, and another transform
    x = random_fr(700, 1 << 15)
    data = gpu.buffer(x)
    ntt = Ntt(gpu, 15)
    coset = CosetShift(gpu, 15, 7)
    nl = len(rnd_sizes)
    batch.add_ntt(ntt, data, inverse=True, lane=nl)
    batch.add_coset(coset, data, lane=nl)
    batch.add_ntt(ntt, data, inverse=False, lane=nl)
    y = random_fr(701, 1 << 12)
    data2 = gpu.buffer(y)
    batch.add_ntt(Ntt(gpu, 12), data2, lane=nl + 1)

    want_chain = cpu.ntt(cpu.coset_shift(cpu.ntt(x, inverse=True), np.array(bn254.words32(7), dtype=np.uint32)))
    want2 = cpu.ntt(y)
    # the same chain one call at a time
    ref = gpu.buffer(x)
    ntt_ref = Ntt(gpu, 15)
    ntt_ref.inverse(gpu, ref)
    CosetShift(gpu, 15, 7).shift(gpu, ref)
    ntt_ref.forward(gpu, ref)
    assert np.array_equal(gpu.read(ref, x.size), want_chain)

    batch.launch()
    gpu.wait()
    assert batch.kernels() > 20
    for (group, out), want in zip(outputs, expected):
        conv = xyzz_to_affine if group == Group.G1 else xyzz_to_affine_g2
        assert np.array_equal(affine_words(conv(gpu.read(out, group.xyzz_words())), group), want)
    assert np.array_equal(gpu.read(data, x.size), want_chain)
    assert np.array_equal(gpu.read(data2, y.size), want2)
    # replay: MSM results identical; the NTT lanes transform their (already transformed) data again
    data.write(x)
    data2.write(y)
    batch.launch()
    gpu.wait()
    for (group, out), want in zip(outputs, expected):
        conv = xyzz_to_affine if group == Group.G1 else xyzz_to_affine_g2
        assert np.array_equal(affine_words(conv(gpu.read(out, group.xyzz_words())), group), want)
    assert np.array_equal(gpu.read(data, x.size), want_chain)
    # and without a graph
    data.write(x)
    batch.run_streams()
    gpu.wait()
    assert np.array_equal(gpu.read(data, x.size), want_chain)


def test_a_plan_belongs_to_one_lane(gpu):
    n = 256
    bases = Msm.upload_bases(gpu, random_points("G1", 1, n))
    s = gpu.buffer(random_fr(2, n))
    plan = Msm(gpu, n, 9)
    batch = Batch(gpu)
    batch.add_msm(plan, bases, s, lane=0)
    with pytest.raises(ZkGpuError, match="one lane only"):
        batch.add_msm(plan, bases, s, lane=1)
    assert bn254.R > 0
