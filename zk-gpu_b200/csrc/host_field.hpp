// Host-side 256-bit modular arithmetic for plan setup (roots of unity, twiddle seeds, n^-1,
// Montgomery constants, fixed-base tables) and for the XYZZ -> affine result conversion.
//
// Replaces the reference's host bignum (src/host.rs:1-115: U256 add/sub/mul/pow/inverse,
// root_of_unity with generator 5, words32 packing) and xyzz_to_affine(_g2) with its Fq2
// helpers (src/msm.rs:345-387). Montgomery radix here is 2^256, matching the device code.
// Never on the hot path: used a few thousand times per plan at most.
#pragma once
#include <cstdint>
#include <cstring>

namespace zkg::host {

using u128 = unsigned __int128;

struct U256 {
  uint64_t v[4];
};

struct Field {
  U256 p;
  uint64_t inv;  // -p^-1 mod 2^64
  U256 r2;       // 2^512 mod p
  U256 one;      // 2^256 mod p
};

inline const Field& fq() {
  static const Field f = {
      {{0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}},
      0x87d20782e4866389ULL,
      {{0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL}},
      {{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}}};
  return f;
}

inline const Field& fr() {
  static const Field f = {
      {{0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL}},
      0xc2e1f593efffffffULL,
      {{0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL}},
      {{0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}}};
  return f;
}

inline bool is_zero(const U256& a) { return (a.v[0] | a.v[1] | a.v[2] | a.v[3]) == 0; }
inline bool eq(const U256& a, const U256& b) { return std::memcmp(&a, &b, sizeof(U256)) == 0; }

inline bool geq(const U256& a, const U256& b) {
  for (int i = 3; i >= 0; i--)
    if (a.v[i] != b.v[i]) return a.v[i] > b.v[i];
  return true;
}

inline U256 sub_raw(const U256& a, const U256& b) {
  U256 r;
  uint64_t borrow = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a.v[i] - b.v[i] - borrow;
    r.v[i] = (uint64_t)d;
    borrow = (uint64_t)(d >> 64) & 1;
  }
  return r;
}

inline U256 add(const U256& a, const U256& b, const Field& f) {
  U256 r;
  u128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (u128)a.v[i] + b.v[i];
    r.v[i] = (uint64_t)c;
    c >>= 64;
  }
  return geq(r, f.p) ? sub_raw(r, f.p) : r;  // p < 2^254: no carry out
}

inline U256 sub(const U256& a, const U256& b, const Field& f) {
  if (geq(a, b)) return sub_raw(a, b);
  U256 d = sub_raw(f.p, b);
  U256 r;
  u128 c = 0;
  for (int i = 0; i < 4; i++) {
    c += (u128)a.v[i] + d.v[i];
    r.v[i] = (uint64_t)c;
    c >>= 64;
  }
  return r;
}

// Montgomery product a * b * 2^-256 mod p.
inline U256 mul(const U256& a, const U256& b, const Field& f) {
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 c = 0;
    for (int j = 0; j < 4; j++) {
      c += (u128)a.v[j] * b.v[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[4] = (uint64_t)c;
    t[5] = (uint64_t)(c >> 64);
    uint64_t m = t[0] * f.inv;
    c = ((u128)m * f.p.v[0] + t[0]) >> 64;
    for (int j = 1; j < 4; j++) {
      c += (u128)m * f.p.v[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[3] = (uint64_t)c;
    t[4] = t[5] + (uint64_t)(c >> 64);
  }
  U256 r = {{t[0], t[1], t[2], t[3]}};
  if (t[4] || geq(r, f.p)) r = sub_raw(r, f.p);
  return r;
}

inline U256 to_mont(const U256& a, const Field& f) { return mul(a, f.r2, f); }
inline U256 from_mont(const U256& a, const Field& f) { return mul(a, U256{{1, 0, 0, 0}}, f); }

// base^e with base in Montgomery form, e a plain 256-bit exponent.
inline U256 pow(const U256& base, const U256& e, const Field& f) {
  U256 acc = f.one;
  for (int bit = 255; bit >= 0; bit--) {
    acc = mul(acc, acc, f);
    if ((e.v[bit / 64] >> (bit % 64)) & 1) acc = mul(acc, base, f);
  }
  return acc;
}

// 1/a by Fermat (src/host.rs:100-102); Montgomery in and out.
inline U256 inverse(const U256& a, const Field& f) { return pow(a, sub_raw(f.p, U256{{2, 0, 0, 0}}), f); }

inline U256 from_words32(const uint32_t* w) {
  U256 r;
  for (int i = 0; i < 4; i++) r.v[i] = (uint64_t)w[2 * i] | ((uint64_t)w[2 * i + 1] << 32);
  return r;
}

inline void words32(const U256& a, uint32_t* w) {
  for (int i = 0; i < 4; i++) {
    w[2 * i] = (uint32_t)a.v[i];
    w[2 * i + 1] = (uint32_t)(a.v[i] >> 32);
  }
}

// Primitive 2^log_n-th root of unity of Fr: 5^((r-1) >> log_n) (src/host.rs:94-98).
// Montgomery form.
inline U256 root_of_unity(uint32_t log_n) {
  const Field& f = fr();
  U256 e = sub_raw(f.p, U256{{1, 0, 0, 0}});
  for (uint32_t s = 0; s < log_n; s++)
    for (int i = 0; i < 4; i++) e.v[i] = (e.v[i] >> 1) | (i < 3 ? e.v[i + 1] << 63 : 0);
  return pow(to_mont(U256{{5, 0, 0, 0}}, f), e, f);
}

// ------------------------------------------------------------------ Fq2 (u^2 = -1)
struct U512 {
  U256 a, b;  // a + b*u
};

inline U512 fq2_mul(const U512& x, const U512& y) {
  const Field& f = fq();
  U256 ac = mul(x.a, y.a, f), bd = mul(x.b, y.b, f);
  U256 ad = mul(x.a, y.b, f), bc = mul(x.b, y.a, f);
  return U512{sub(ac, bd, f), add(ad, bc, f)};
}

// 1/(a + bu) = (a - bu) / (a^2 + b^2)
inline U512 fq2_inverse(const U512& x) {
  const Field& f = fq();
  U256 nrm = add(mul(x.a, x.a, f), mul(x.b, x.b, f), f);
  U256 inv = inverse(nrm, f);
  return U512{mul(x.a, inv, f), sub(U256{{0, 0, 0, 0}}, mul(x.b, inv, f), f)};
}

}  // namespace zkg::host
