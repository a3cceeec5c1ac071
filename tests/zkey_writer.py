"""Writes Groth16 proving keys in snarkjs's .zkey layout (test infrastructure: the tests build
small keys with it and read them back through zkg_zkey_*).

Layout (little-endian; the reader's comment in zk-gpu_b200/csrc/zkey.hpp states it in full):
"zkey", version 1, section count; sections (type u32, size u64, bytes): 1 protocol (1 =
Groth16); 2 header (n8q, q, n8r, r, nVars, nPublic, domainSize, alpha1, beta1, beta2, gamma2,
delta1, delta2); 3 IC, 4 coefficients, 5 A, 6 B1, 7 B2, 8 C, 9 H, 10 contributions. Points in
Montgomery form with R = 2^256 (16 words per G1 point, 32 per G2), infinity as zeros.
"""
from __future__ import annotations

import struct

import numpy as np

from oracle import bn254, cpu
from zk_gpu.synthetic import uniform_scalars


def _section(kind: int, body: bytes) -> bytes:
    return struct.pack("<IQ", kind, len(body)) + body


def _int_bytes(v: int) -> bytes:
    return v.to_bytes(32, "little")


def random_points(group: str, n: int, seed: int, infinity_every: int = 0) -> np.ndarray:
    """n points [k]G in Montgomery-2^256 words; every `infinity_every`-th one at infinity."""
    aw = 16 if group == "G1" else 32
    pts = cpu.generator_multiples(group, uniform_scalars(n, seed), mont256=True).reshape(n, aw)
    if infinity_every:
        pts[::infinity_every] = 0
    return pts.reshape(-1)


def build(n_vars: int, n_public: int, domain_size: int, seed: int = 1, infinity_every: int = 0,
          protocol: int = 1, q: int = bn254.Q, extra_sections: bool = True) -> tuple[bytes, dict]:
    """A key image and the point sections it holds (section id -> words)."""
    pts = {
        3: random_points("G1", n_public + 1, seed + 3, infinity_every),
        5: random_points("G1", n_vars, seed + 5, infinity_every),
        6: random_points("G1", n_vars, seed + 6, infinity_every),
        7: random_points("G2", n_vars, seed + 7, infinity_every),
        8: random_points("G1", n_vars - n_public - 1, seed + 8, infinity_every),
        9: random_points("G1", domain_size, seed + 9, infinity_every),
    }
    g1 = random_points("G1", 3, seed + 11).tobytes()
    g2 = random_points("G2", 3, seed + 12).tobytes()
    header = (struct.pack("<I", 32) + _int_bytes(q) + struct.pack("<I", 32) + _int_bytes(bn254.R) +
              struct.pack("<III", n_vars, n_public, domain_size) +
              g1[0:64] + g1[64:128] + g2[0:128] + g2[128:256] + g1[128:192] + g2[256:384])
    sections = [_section(1, struct.pack("<I", protocol)), _section(2, header), _section(3, pts[3].tobytes())]
    if extra_sections:
        sections.append(_section(4, struct.pack("<I", 0)))  # no constraint coefficients
    sections += [_section(k, pts[k].tobytes()) for k in (5, 6, 7, 8, 9)]
    if extra_sections:
        sections.append(_section(10, b"\x00" * 64))
    image = b"zkey" + struct.pack("<II", 1, len(sections)) + b"".join(sections)
    return image, pts
