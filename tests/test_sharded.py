"""MSM over a key sharded across ranks (zk_gpu.sharded): the host XYZZ addition against the
oracle's group law, the rank-ordered gather and sum on world_size 2 gloo ranks on the CPU (each
rank's partial made by the oracle there), and on the GPU shards of one key run one after another
in one process, summed, against the oracle's MSM of the whole key."""
import os

import numpy as np
import pytest

from common import random_fr, random_points
from oracle import bn254, cpu
from zk_gpu import Group, Msm, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.sharded import shard_bounds, xyzz_sum

Q, R = bn254.Q, bn254.R
MONT = pow(2, 256, Q)


def to_xyzz_words(group: str, affine_words_: np.ndarray) -> np.ndarray:
    """Plain affine words (zeros = infinity) -> XYZZ words with ZZ = ZZZ = 1, Montgomery 2^256."""
    w = [bn254.from_words32(affine_words_[8 * k: 8 * k + 8]) for k in range(affine_words_.size // 8)]
    if not any(w):
        return np.zeros(2 * affine_words_.size, dtype=np.uint32)
    mont = [v * MONT % Q for v in w]
    one = [MONT] + ([0] if group == "G2" else [])
    return np.array([x for v in mont + one + one for x in bn254.words32(v)], dtype=np.uint32)


def from_xyzz(group: str, words: np.ndarray) -> np.ndarray:
    grp = Group.G1 if group == "G1" else Group.G2
    conv = xyzz_to_affine if grp == Group.G1 else xyzz_to_affine_g2
    return affine_words(conv(words), grp)


@pytest.mark.parametrize("group", ["G1", "G2"])
def test_host_addition_matches_oracle(group):
    aw = 16 if group == "G1" else 32
    grp = Group.G1 if group == "G1" else Group.G2
    pts = random_points(group, 60, 3)
    p, q = pts[:aw], pts[aw: 2 * aw]
    neg_p = cpu.scalar_mul(group, p, np.array(bn254.words32(R - 1), dtype=np.uint32))
    zero = np.zeros(aw, dtype=np.uint32)
    two_p = cpu.scalar_mul(group, p, np.array(bn254.words32(2), dtype=np.uint32))
    p_plus_q = cpu.msm(group, np.concatenate([p, q]), np.array(bn254.words32(1) * 2, dtype=np.uint32))
    for a, b, want in [(p, q, p_plus_q), (p, p, two_p), (p, neg_p, zero), (p, zero, p), (zero, q, q), (zero, zero, zero)]:
        got = xyzz_sum(grp, [to_xyzz_words(group, a), to_xyzz_words(group, b)])
        assert np.array_equal(from_xyzz(group, got), want)


def _gloo_rank(rank, world, port, group, n, result):
    import torch.distributed as dist

    from zk_gpu.sharded import gather_partials

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        bases = random_points(group, 70, n)
        s = random_fr(71, n)
        aw = 16 if group == "G1" else 32
        lo, hi = shard_bounds(n, rank, world)
        # the oracle stands in for this rank's GPU MSM over its shard
        local = to_xyzz_words(group, cpu.msm(group, bases[lo * aw: hi * aw], s[8 * lo: 8 * hi]))
        total = xyzz_sum(Group.G1 if group == "G1" else Group.G2, gather_partials(local))
        result[rank] = from_xyzz(group, total).tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("group", ["G1", "G2"])
def test_two_ranks_sum_to_the_whole_msm(group):
    import multiprocessing as mp
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    n = 301
    with ctx.Manager() as m:
        result = m.dict()
        procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, group, n, result)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        want = cpu.msm(group, random_points(group, 70, n), random_fr(71, n))
        for r in range(2):
            assert np.array_equal(np.array(result[r], dtype=np.uint32), want), r


def test_shard_bounds_cover_the_key():
    for n, world in [(10, 3), (1 << 20, 8), (5, 8)]:
        spans = [shard_bounds(n, r, world) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == n
        assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
        assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1


@pytest.mark.gpu
@pytest.mark.parametrize("group", ["G1", "G2"])
def test_shards_on_one_gpu_sum_to_the_whole_msm(gpu, group):
    grp = Group.G1 if group == "G1" else Group.G2
    aw = grp.affine_words()
    n, world = 1 << 13, 3
    bases = random_points(group, 80, n)
    s = random_fr(81, n)
    partials = []
    for r in range(world):
        lo, hi = shard_bounds(n, r, world)
        msm = Msm.for_group(gpu, grp, hi - lo, Msm.default_window(n))
        out = msm.run(gpu, Msm.upload_bases(gpu, bases[lo * aw: hi * aw]), gpu.buffer(s[8 * lo: 8 * hi]))
        partials.append(gpu.read(out, grp.xyzz_words()))
    assert np.array_equal(from_xyzz(group, xyzz_sum(grp, partials)), cpu.msm(group, bases, s))
