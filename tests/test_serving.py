"""The proving-request server: every request's outputs are the same alone (plain path, one
request at a time) and in a concurrent mix (served path: lanes, graphs, continuous batching),
and they match the oracle; admission under a tight HBM budget evicts idle slots and stays
correct."""
import numpy as np
import pytest

from common import random_fr
from oracle import bn254, cpu
from zk_gpu import Group, Msm, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.serving import ProofInputs, Server
from zk_gpu.synthetic import uniform_scalars

pytestmark = pytest.mark.gpu
R = bn254.R
G = 7
KEY_N = 1 << 12


@pytest.fixture(scope="module")
def key(gpu):
    g1 = cpu.generator_multiples("G1", uniform_scalars(KEY_N, 71))
    g2 = cpu.generator_multiples("G2", uniform_scalars(KEY_N, 72))
    return g1, g2, Msm.upload_bases(gpu, g1), Msm.upload_bases(gpu, g2)


def make_request(log_m, seed):
    m = 1 << log_m
    req = ProofInputs(log_m)
    g1 = [random_fr(seed + j, m) for j in range(3)]
    g1[2] = g1[2][: 8 * (m - 1024)]
    polys = [random_fr(seed + 10 + j, 2 * m) for j in range(3)]
    return req.fill(g1, random_fr(seed + 5, m), polys)


def words_to_ints(w):
    return [bn254.from_words32(w[8 * i: 8 * i + 8]) for i in range(w.size // 8)]


def oracle_outputs(key, req):
    g1_plain, g2_plain = key[0], key[1]
    m, N = req.m, req.N
    pts = []
    for j in range(3):
        cnt = req.g1_counts[j]
        pts.append(cpu.msm("G1", g1_plain[: 16 * cnt], req.g1[j].array[: 8 * cnt]))
    pts.append(cpu.msm("G2", g2_plain[: 32 * m], req.g2.array))
    g = np.array(bn254.words32(G), dtype=np.uint32)
    ev = [cpu.ntt(cpu.coset_shift(cpu.ntt(p.array, True), g)) for p in req.polys]
    a, b, c = (words_to_ints(e) for e in ev)
    zinv = pow((pow(G, N, R) - 1) % R, R - 2, R)
    h = np.array([w for x, y, z in zip(a, b, c) for w in bn254.words32((x * y - z) * zinv % R)], dtype=np.uint32)
    ginv = np.array(bn254.words32(pow(G, R - 2, R)), dtype=np.uint32)
    return pts, cpu.coset_shift(cpu.ntt(h, True), ginv)


def affine_points(words):
    out = [affine_words(xyzz_to_affine(words[32 * j: 32 * j + 32])) for j in range(3)]
    out.append(affine_words(xyzz_to_affine_g2(words[96:160]), Group.G2))
    return out


def run_plain(gpu, key, reqs):
    server = Server(gpu, plain=True, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    outs = []
    for r in reqs:
        server.wait(server.submit(r))
        outs.append((affine_points(r.points()), r.h()))
    server.close()
    return outs


def same_points(a, b):
    """XYZZ words are not canonical (the bucket order inside a sort is not fixed); the affine
    reading is."""
    return all(np.array_equal(x, y) for x, y in zip(a, b))


def test_results_are_the_same_alone_and_in_the_mix(gpu, key):
    sizes = [11, 12, 11, 12, 12, 11, 11, 12]
    alone = run_plain(gpu, key, [make_request(lm, 1000 + 37 * i) for i, lm in enumerate(sizes)])
    reqs = [make_request(lm, 1000 + 37 * i) for i, lm in enumerate(sizes)]
    server = Server(gpu, lanes=4, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    ids = [server.submit(r) for r in reqs]  # all at once: they queue and overlap
    for rid in ids:
        server.wait(rid)
    stats = server.stats()
    assert stats["completed"] == len(reqs) and stats["slots_created"] >= 2
    for i, r in enumerate(reqs):
        assert same_points(affine_points(r.points()), alone[i][0]), f"request {i}: MSM results differ in the mix"
        assert np.array_equal(r.h(), alone[i][1]), f"request {i}: h differs in the mix"
    for i in (0, 1):
        pts, h = oracle_outputs(key, reqs[i])
        got = affine_points(reqs[i].points())
        for j in range(4):
            assert np.array_equal(got[j], pts[j]), f"request {i}: MSM {j} differs from the oracle"
        assert np.array_equal(reqs[i].h(), h), f"request {i}: h differs from the oracle"
    server.close()


def test_tight_budget_evicts_and_stays_correct(gpu, key):
    reqs = [make_request(lm, 5000 + 11 * i) for i, lm in enumerate([11, 12, 11, 12])]
    alone = run_plain(gpu, key, [make_request(lm, 5000 + 11 * i) for i, lm in enumerate([11, 12, 11, 12])])
    server = Server(gpu, lanes=2, hbm_budget_bytes=1 << 20, coset_g=G)  # below one slot: one at a time
    server.add_key(KEY_N, key[2], key[3])
    for r in reqs:
        server.wait(server.submit(r))
    stats = server.stats()
    assert stats["slots_evicted"] >= 2
    for i, r in enumerate(reqs):
        assert same_points(affine_points(r.points()), alone[i][0]) and np.array_equal(r.h(), alone[i][1])
    server.close()


def test_rejects_requests_without_a_key(gpu, key):
    from zk_gpu import ZkGpuError
    server = Server(gpu, lanes=2, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    with pytest.raises(ZkGpuError, match="no resident proving key"):
        server.submit(ProofInputs(13))
    server.close()


def test_reserved_slots_serve_a_burst_without_new_slots(gpu, key):
    """reserve() makes idle slots ahead of time; a burst of that many same-size requests runs on
    them without making more, and the results match the plain path."""
    reqs = [make_request(11, 7000 + 13 * i) for i in range(3)]
    alone = run_plain(gpu, key, [make_request(11, 7000 + 13 * i) for i in range(3)])
    server = Server(gpu, lanes=3, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    server.reserve(11, 3)
    server.reserve(11, 2)  # already held: no-op
    before = server.stats()
    assert before["slots"] == 3 and before["slots_created"] == 3 and before["build_ms"] > 0
    ids = [server.submit(r) for r in reqs]
    for rid in ids:
        server.wait(rid)
    after = server.stats()
    assert after["slots_created"] == 3 and after["completed"] == 3
    for i, r in enumerate(reqs):
        assert same_points(affine_points(r.points()), alone[i][0]) and np.array_equal(r.h(), alone[i][1])
    server.close()


def test_busy_slots_of_a_size_are_waited_for(gpu, key):
    """A size that has its reserved slots (at least two) all busy does not get another built:
    its next requests wait for them (a build under load costs more than the wait); an unreserved
    size gets at most two. All requests complete with the plain path's results."""
    sizes = [11] * 6 + [12] * 5
    reqs = [make_request(lm, 9000 + 19 * i) for i, lm in enumerate(sizes)]
    alone = run_plain(gpu, key, [make_request(lm, 9000 + 19 * i) for i, lm in enumerate(sizes)])
    server = Server(gpu, lanes=6, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    server.reserve(11, 2)
    ids = [server.submit(r) for r in reqs]  # all at once: more same-size requests than slots
    for rid in ids:
        server.wait(rid)
    stats = server.stats()
    assert stats["completed"] == len(reqs)
    assert stats["slots_created"] == 4, stats  # two reserved for 2^11, two built for 2^12
    for i, r in enumerate(reqs):
        assert same_points(affine_points(r.points()), alone[i][0]) and np.array_equal(r.h(), alone[i][1]), i
    server.close()


def test_requests_with_slots_pass_one_whose_slot_is_being_made(gpu, key):
    """A request that needs a new slot does not hold back later requests whose slots exist: all
    complete, with the plain path's results."""
    sizes = [12, 11, 11, 11]
    reqs = [make_request(lm, 8000 + 17 * i) for i, lm in enumerate(sizes)]
    alone = run_plain(gpu, key, [make_request(lm, 8000 + 17 * i) for i, lm in enumerate(sizes)])
    server = Server(gpu, lanes=4, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    server.reserve(11, 3)
    ids = [server.submit(r) for r in reqs]
    for rid in ids:
        server.wait(rid)
    stats = server.stats()
    assert stats["slots_created"] == 4 and stats["completed"] == 4
    for i, r in enumerate(reqs):
        assert same_points(affine_points(r.points()), alone[i][0]) and np.array_equal(r.h(), alone[i][1])
    server.close()


def test_reserve_checks_the_budget_and_the_keys(gpu, key):
    from zk_gpu import ZkGpuError
    server = Server(gpu, lanes=2, hbm_budget_bytes=1 << 20, coset_g=G)
    server.add_key(KEY_N, key[2], key[3])
    with pytest.raises(ZkGpuError, match="does not fit the HBM budget"):
        server.reserve(11, 1)
    with pytest.raises(ZkGpuError, match="no resident proving key"):
        server.reserve(13, 1)
    assert server.stats()["bytes_used"] == 0
    server.close()
