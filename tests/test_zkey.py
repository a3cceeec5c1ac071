"""snarkjs .zkey ingestion (zkg_zkey_*): the host parser on any machine, and MSMs over uploaded
point sections against the oracle on the GPU (the reference's tests/properties.rs:222-246 and
tests/g2.rs:89-111 feed Montgomery-2^256 points the same way)."""
import struct

import numpy as np
import pytest

import zkey_writer
from common import random_fr
from oracle import bn254, cpu
from zk_gpu import Group, Msm, ZkGpuError, xyzz_to_affine, xyzz_to_affine_g2
from zk_gpu.msm import affine_words
from zk_gpu.zkey import A, B1, B2, C, H, IC, Zkey


def test_header_and_points_round_trip():
    image, pts = zkey_writer.build(n_vars=40, n_public=3, domain_size=64, infinity_every=7)
    z = Zkey(image)
    assert z.header() == {"protocol": 1, "n_vars": 40, "n_public": 3, "domain_size": 64}
    for section, group, count in [(IC, Group.G1, 4), (A, Group.G1, 40), (B1, Group.G1, 40), (B2, Group.G2, 40),
                                  (C, Group.G1, 36), (H, Group.G1, 64)]:
        words, g = z.points(section)
        assert g == group and words.size == count * group.affine_words()
        assert np.array_equal(words, pts[section]), section


def test_without_optional_sections():
    image, pts = zkey_writer.build(n_vars=5, n_public=1, domain_size=8, extra_sections=False)
    assert np.array_equal(Zkey(image).points(H)[0], pts[H])


def _patched(image: bytes, offset: int, data: bytes) -> bytes:
    return image[:offset] + data + image[offset + len(data):]


def test_malformed_keys_are_rejected():
    image, _ = zkey_writer.build(n_vars=6, n_public=1, domain_size=8)
    cases = [
        (b"zkez" + image[4:], "not a zkey file"),
        (image[:8] + struct.pack("<I", 99) + image[12:], "zkey truncated|truncated"),
        (image[:-10], "truncated"),
        (_patched(image, 4, struct.pack("<I", 2)), "version 2 is not supported"),
        (zkey_writer.build(6, 1, 8, protocol=2)[0], "protocol 2 is not Groth16"),
        (zkey_writer.build(6, 1, 8, q=bn254.R)[0], "base field is not BN254"),
        (zkey_writer.build(6, 1, 7)[0], "domainSize is not a power of two"),
    ]
    for data, msg in cases:
        with pytest.raises(ZkGpuError, match=msg):
            Zkey(data)
    # a coordinate at q (not reduced)
    words = np.frombuffer(image, dtype=np.uint8).copy()
    sec5 = image.index(struct.pack("<IQ", 5, 6 * 64)) + 12
    words[sec5: sec5 + 32] = np.frombuffer(bn254.Q.to_bytes(32, "little"), dtype=np.uint8)
    with pytest.raises(ZkGpuError, match="is not below q"):
        Zkey(words.tobytes())
    # a section whose size does not match the header
    bad = _patched(image, sec5 - 8, struct.pack("<Q", 5 * 64))
    with pytest.raises(ZkGpuError, match="zkey section 5 holds|truncated"):
        Zkey(bad)
    z = Zkey(image)
    with pytest.raises(ZkGpuError, match="not a point section"):
        z.points(4)


@pytest.mark.gpu
@pytest.mark.parametrize("section", [A, B1, B2, C, H])
def test_msm_over_uploaded_sections_matches_oracle(gpu, section):
    """Each point section uploaded as resident bases, including points at infinity, and an MSM
    over it equal to the oracle's MSM of the same Montgomery-2^256 points."""
    image, pts = zkey_writer.build(n_vars=700, n_public=5, domain_size=1024, infinity_every=13, seed=31)
    z = Zkey(image)
    bases = z.upload(gpu, section)
    words, group = z.points(section)
    n = words.size // group.affine_words()
    s = random_fr(40 + section, n)
    msm = Msm.for_group(gpu, group, n, Msm.default_window(n))
    out = gpu.read(msm.run(gpu, bases, gpu.buffer(s)), group.xyzz_words())
    conv = xyzz_to_affine if group == Group.G1 else xyzz_to_affine_g2
    got = affine_words(conv(out), group)
    gname = "G1" if group == Group.G1 else "G2"
    assert np.array_equal(got, cpu.msm(gname, pts[section], s, mont256=True)), section
