"""host: 256-bit modular helpers for set-up work on the CPU (src/host.rs:1-115).

Integers instead of [u64; 4]; `montgomery_r` returns this library's radix 2^256 mod m (the
reference's WGSL kernels use 2^260). Never used on the device path.
"""
from __future__ import annotations

FQ = 0x30644E72E131A029B85045B68181585D97816A916871CA8D3C208C16D87CFD47  # src/field.rs:18
FR = 0x30644E72E131A029B85045B68181585D2833E84879B9709143E1F593F0000001  # src/field.rs:20


def add_mod(a: int, b: int, m: int) -> int:
    return (a + b) % m


def sub_mod(a: int, b: int, m: int) -> int:
    return (a - b) % m


def mul_mod(a: int, b: int, m: int) -> int:
    return a * b % m


def pow_mod(base: int, exp: int, m: int) -> int:
    return pow(base, exp, m)


def inverse(x: int, m: int) -> int:
    """By Fermat (src/host.rs:100-102)."""
    return pow(x, m - 2, m)


def montgomery_r(m: int) -> int:
    """R mod m for this library's Montgomery radix R = 2^256."""
    return (1 << 256) % m


def root_of_unity(log_n: int) -> int:
    """Primitive 2^log_n-th root of unity of Fr, generator 5 (src/host.rs:94-98)."""
    return pow(5, (FR - 1) >> log_n, FR)


def from_montgomery(x: int, m: int) -> int:
    """x * R^-1 mod m (src/host.rs:113-115)."""
    return x * inverse(montgomery_r(m), m) % m


def words32(x: int) -> list[int]:
    """Integer -> 8 little-endian u32 words (src/host.rs:104-106)."""
    return [(x >> (32 * i)) & 0xFFFFFFFF for i in range(8)]


def from_words32(w) -> int:
    """8 little-endian u32 words -> integer (src/host.rs:108-110)."""
    return sum(int(w[i]) << (32 * i) for i in range(8))


def from_u64s(limbs) -> int:
    """[u64; 4] little-endian limbs -> integer."""
    return sum(int(v) << (64 * i) for i, v in enumerate(limbs))
