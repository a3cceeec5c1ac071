// BN254 base field Fq and scalar field Fr on sm_100a: 8 x 32-bit limbs, Montgomery radix
// R = 2^256, products on the integer multiply-add pipe (mad.wide.u32) with PTX carry chains
// (add.cc / addc) for the accumulation. No tensor cores: this is exact modular integer
// arithmetic.
//
// Replaces the reference's generated WGSL field code (src/field.rs:55-181: 20 x 13-bit limbs,
// R = 2^260, deferred carries). Memory format is unchanged: 8 little-endian u32 words per
// element (src/field.rs:63-93). Values in registers and in memory are always fully reduced
// (< p), so equality and zero tests are word compares.
#pragma once
#include <cstdint>

namespace zkg {

// Modulus parameters. INV = -p^-1 mod 2^32; ONE = 2^256 mod p (Montgomery one);
// R2 = 2^512 mod p (to_montgomery multiplier).
struct FqParams {
  static constexpr bool kCompact = false;
  static constexpr bool kPairs = false;
  static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du, P3 = 0x97816a91u;
  static constexpr uint32_t P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xe4866389u;
  static constexpr uint32_t ONE0 = 0xc58f0d9du, ONE1 = 0xd35d438du, ONE2 = 0xf5c70b3du, ONE3 = 0x0a78eb28u;
  static constexpr uint32_t ONE4 = 0x7879462cu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
};

struct FrParams {
  static constexpr bool kCompact = false;
  static constexpr bool kPairs = false;
  static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u, P3 = 0x2833e848u;
  static constexpr uint32_t P4 = 0x8181585du, P5 = 0xb85045b6u, P6 = 0xe131a029u, P7 = 0x30644e72u;
  static constexpr uint32_t INV = 0xefffffffu;
  static constexpr uint32_t ONE0 = 0x4ffffffbu, ONE1 = 0xac96341cu, ONE2 = 0x9f60cd29u, ONE3 = 0x36fc7695u;
  static constexpr uint32_t ONE4 = 0x7879462eu, ONE5 = 0x666ea36fu, ONE6 = 0x9a07df2fu, ONE7 = 0x0e0a77c1u;
};

// Same field, products through one out-of-line function instead of inlined copies. Kernels
// where few warps run long serial chains (merge, bucket reduction, window combination) use
// it: a fully inlined point addition is thousands of instructions, and a lone warp walking
// through straight-line code that size waits on instruction fetch rather than arithmetic.
struct FqCompactParams : FqParams {
  static constexpr bool kCompact = true;
};

// Compact, and independent products go two per call (mul2): shorter dependency waits for a
// lone thread, more registers per thread.
struct FqCompactPairParams : FqParams {
  static constexpr bool kCompact = true;
  static constexpr bool kPairs = true;
};

template <class P>
struct Fp {
  uint32_t w[8];

  __device__ __forceinline__ static Fp zero() {
    Fp r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.w[i] = 0;
    return r;
  }
  __device__ __forceinline__ static Fp one() {
    Fp r;
    r.w[0] = P::ONE0; r.w[1] = P::ONE1; r.w[2] = P::ONE2; r.w[3] = P::ONE3;
    r.w[4] = P::ONE4; r.w[5] = P::ONE5; r.w[6] = P::ONE6; r.w[7] = P::ONE7;
    return r;
  }
  __device__ __forceinline__ bool is_zero() const {
    uint32_t x = w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7];
    return x == 0;
  }
  __device__ __forceinline__ bool operator==(const Fp& o) const {
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) x |= w[i] ^ o.w[i];
    return x == 0;
  }
  __device__ __forceinline__ bool operator!=(const Fp& o) const { return !(*this == o); }
};

using Fq = Fp<FqParams>;
using Fr = Fp<FrParams>;
using FqC = Fp<FqCompactParams>;
using FqCP = Fp<FqCompactPairParams>;

// ------------------------------------------------------------------ add / sub

// r = a + b mod p. Both < p < 2^254, so a + b < 2^255 never carries out of 8 words.
template <class P>
__device__ __forceinline__ Fp<P> operator+(const Fp<P>& a, const Fp<P>& b) {
  Fp<P> s, d;
  uint32_t borrow;
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=&r"(s.w[0]), "=&r"(s.w[1]), "=&r"(s.w[2]), "=&r"(s.w[3]), "=&r"(s.w[4]), "=&r"(s.w[5]), "=&r"(s.w[6]),
        "=&r"(s.w[7])
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(a.w[4]), "r"(a.w[5]), "r"(a.w[6]), "r"(a.w[7]),
        "r"(b.w[0]), "r"(b.w[1]), "r"(b.w[2]), "r"(b.w[3]), "r"(b.w[4]), "r"(b.w[5]), "r"(b.w[6]), "r"(b.w[7]));
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=&r"(d.w[0]), "=&r"(d.w[1]), "=&r"(d.w[2]), "=&r"(d.w[3]), "=&r"(d.w[4]), "=&r"(d.w[5]), "=&r"(d.w[6]),
        "=&r"(d.w[7]), "=&r"(borrow)
      : "r"(s.w[0]), "r"(s.w[1]), "r"(s.w[2]), "r"(s.w[3]), "r"(s.w[4]), "r"(s.w[5]), "r"(s.w[6]), "r"(s.w[7]),
        "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5), "n"(P::P6), "n"(P::P7));
  // borrow = 0xffffffff when s < p: keep s; otherwise take s - p.
  Fp<P> r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = (s.w[i] & borrow) | (d.w[i] & ~borrow);
  return r;
}

// r = a - b mod p: subtract, then add p back under the borrow mask.
template <class P>
__device__ __forceinline__ Fp<P> operator-(const Fp<P>& a, const Fp<P>& b) {
  Fp<P> d, r;
  uint32_t borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=&r"(d.w[0]), "=&r"(d.w[1]), "=&r"(d.w[2]), "=&r"(d.w[3]), "=&r"(d.w[4]), "=&r"(d.w[5]), "=&r"(d.w[6]),
        "=&r"(d.w[7]), "=&r"(borrow)
      : "r"(a.w[0]), "r"(a.w[1]), "r"(a.w[2]), "r"(a.w[3]), "r"(a.w[4]), "r"(a.w[5]), "r"(a.w[6]), "r"(a.w[7]),
        "r"(b.w[0]), "r"(b.w[1]), "r"(b.w[2]), "r"(b.w[3]), "r"(b.w[4]), "r"(b.w[5]), "r"(b.w[6]), "r"(b.w[7]));
  asm("add.cc.u32  %0, %8, %16;\n\t"
      "addc.cc.u32 %1, %9, %17;\n\t"
      "addc.cc.u32 %2, %10, %18;\n\t"
      "addc.cc.u32 %3, %11, %19;\n\t"
      "addc.cc.u32 %4, %12, %20;\n\t"
      "addc.cc.u32 %5, %13, %21;\n\t"
      "addc.cc.u32 %6, %14, %22;\n\t"
      "addc.u32    %7, %15, %23;"
      : "=&r"(r.w[0]), "=&r"(r.w[1]), "=&r"(r.w[2]), "=&r"(r.w[3]), "=&r"(r.w[4]), "=&r"(r.w[5]), "=&r"(r.w[6]),
        "=&r"(r.w[7])
      : "r"(d.w[0]), "r"(d.w[1]), "r"(d.w[2]), "r"(d.w[3]), "r"(d.w[4]), "r"(d.w[5]), "r"(d.w[6]), "r"(d.w[7]),
        "r"(P::P0 & borrow), "r"(P::P1 & borrow), "r"(P::P2 & borrow), "r"(P::P3 & borrow), "r"(P::P4 & borrow),
        "r"(P::P5 & borrow), "r"(P::P6 & borrow), "r"(P::P7 & borrow));
  return r;
}

template <class P>
__device__ __forceinline__ Fp<P> neg(const Fp<P>& a) {
  return Fp<P>::zero() - a;
}

template <class P>
__device__ __forceinline__ Fp<P> dbl(const Fp<P>& a) {
  return a + a;
}

// ------------------------------------------------------------------ Montgomery product
//
// Coarsely integrated operand scanning with 32x32 -> 64-bit products. On sm_100a the wide
// multiply (mad.wide.u32, one instruction for both halves of a product plus a 32-bit addend)
// issues at the same rate as mul.hi alone, so a row x*v costs 8 wide multiply-adds on the
// integer multiply pipe and one 8-long add.cc chain on the integer add pipe, instead of 8 low
// plus 8 high multiply-adds: 2/3 of the multiply-pipe time of the lo/hi formulation, and the 8
// products of a row are independent (a short dependency chain for single-thread latency).
//
// Row i (product or reduction) with d_j = x * v_j + t[i+j] < 2^64:
//   t[i] = lo(d_0),  t[i+j] = lo(d_j) + hi(d_{j-1}) + carry (j = 1..7),
//   t[i+8] (+)= hi(d_7) + carry.
// The running value stays below 2^288 because p < 2^254, so word i+8 never carries out.

// Product row: t[i+8] is fresh (never written before this row).
#define ZKG_WIDE_CHAIN_FRESH(t, i, d)                                                            \
  asm("add.cc.u32  %0, %8, %9;\n\t"                                                              \
      "addc.cc.u32 %1, %10, %11;\n\t"                                                            \
      "addc.cc.u32 %2, %12, %13;\n\t"                                                            \
      "addc.cc.u32 %3, %14, %15;\n\t"                                                            \
      "addc.cc.u32 %4, %16, %17;\n\t"                                                            \
      "addc.cc.u32 %5, %18, %19;\n\t"                                                            \
      "addc.cc.u32 %6, %20, %21;\n\t"                                                            \
      "addc.u32    %7, %22, 0;"                                                                   \
      : "=&r"(t[i + 1]), "=&r"(t[i + 2]), "=&r"(t[i + 3]), "=&r"(t[i + 4]), "=&r"(t[i + 5]),      \
        "=&r"(t[i + 6]), "=&r"(t[i + 7]), "=&r"(t[i + 8])                                         \
      : "r"((uint32_t)d[1]), "r"((uint32_t)(d[0] >> 32)), "r"((uint32_t)d[2]),                    \
        "r"((uint32_t)(d[1] >> 32)), "r"((uint32_t)d[3]), "r"((uint32_t)(d[2] >> 32)),            \
        "r"((uint32_t)d[4]), "r"((uint32_t)(d[3] >> 32)), "r"((uint32_t)d[5]),                    \
        "r"((uint32_t)(d[4] >> 32)), "r"((uint32_t)d[6]), "r"((uint32_t)(d[5] >> 32)),            \
        "r"((uint32_t)d[7]), "r"((uint32_t)(d[6] >> 32)), "r"((uint32_t)(d[7] >> 32)))

// Reduction row: t[i+8] holds the product row's top word and accumulates.
#define ZKG_WIDE_CHAIN_ACC(t, i, d)                                                              \
  asm("add.cc.u32  %0, %8, %9;\n\t"                                                              \
      "addc.cc.u32 %1, %10, %11;\n\t"                                                            \
      "addc.cc.u32 %2, %12, %13;\n\t"                                                            \
      "addc.cc.u32 %3, %14, %15;\n\t"                                                            \
      "addc.cc.u32 %4, %16, %17;\n\t"                                                            \
      "addc.cc.u32 %5, %18, %19;\n\t"                                                            \
      "addc.cc.u32 %6, %20, %21;\n\t"                                                            \
      "addc.u32    %7, %7, %22;"                                                                  \
      : "=&r"(t[i + 1]), "=&r"(t[i + 2]), "=&r"(t[i + 3]), "=&r"(t[i + 4]), "=&r"(t[i + 5]),      \
        "=&r"(t[i + 6]), "=&r"(t[i + 7]), "+r"(t[i + 8])                                          \
      : "r"((uint32_t)d[1]), "r"((uint32_t)(d[0] >> 32)), "r"((uint32_t)d[2]),                    \
        "r"((uint32_t)(d[1] >> 32)), "r"((uint32_t)d[3]), "r"((uint32_t)(d[2] >> 32)),            \
        "r"((uint32_t)d[4]), "r"((uint32_t)(d[3] >> 32)), "r"((uint32_t)d[5]),                    \
        "r"((uint32_t)(d[4] >> 32)), "r"((uint32_t)d[6]), "r"((uint32_t)(d[5] >> 32)),            \
        "r"((uint32_t)d[7]), "r"((uint32_t)(d[6] >> 32)), "r"((uint32_t)(d[7] >> 32)))

// Returns a * b * 2^-256 mod p.
template <class P>
__device__ __forceinline__ Fp<P> mont_mul_inline(const Fp<P>& a, const Fp<P>& b) {
  constexpr uint32_t q[8] = {P::P0, P::P1, P::P2, P::P3, P::P4, P::P5, P::P6, P::P7};
  uint32_t t[17];
#pragma unroll
  for (int i = 0; i < 8; i++) t[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    uint64_t d[8];
#pragma unroll
    for (int j = 0; j < 8; j++) d[j] = (uint64_t)a.w[j] * b.w[i] + t[i + j];
    t[i] = (uint32_t)d[0];
    ZKG_WIDE_CHAIN_FRESH(t, i, d);
    const uint32_t m = t[i] * P::INV;  // clears word i
#pragma unroll
    for (int j = 0; j < 8; j++) d[j] = (uint64_t)m * q[j] + t[i + j];
    ZKG_WIDE_CHAIN_ACC(t, i, d);
  }
  // t[8..15] < 2p: one conditional subtraction.
  Fp<P> s, d;
#pragma unroll
  for (int i = 0; i < 8; i++) s.w[i] = t[8 + i];
  uint32_t borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=&r"(d.w[0]), "=&r"(d.w[1]), "=&r"(d.w[2]), "=&r"(d.w[3]), "=&r"(d.w[4]), "=&r"(d.w[5]), "=&r"(d.w[6]),
        "=&r"(d.w[7]), "=&r"(borrow)
      : "r"(s.w[0]), "r"(s.w[1]), "r"(s.w[2]), "r"(s.w[3]), "r"(s.w[4]), "r"(s.w[5]), "r"(s.w[6]), "r"(s.w[7]),
        "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5), "n"(P::P6), "n"(P::P7));
  Fp<P> r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = (s.w[i] & borrow) | (d.w[i] & ~borrow);
  return r;
}

// Add chains for rows of plain mul.wide products (no 64-bit addend to assemble): one chain for
// the low halves and one for the high halves one word up. t[i+8] is fresh in a product row and
// accumulates in a reduction row.
#define ZKG_ADD_LO_FRESH(t, i, d)                                                                \
  asm("add.cc.u32  %0, %0, %9;\n\t"                                                              \
      "addc.cc.u32 %1, %1, %10;\n\t"                                                             \
      "addc.cc.u32 %2, %2, %11;\n\t"                                                             \
      "addc.cc.u32 %3, %3, %12;\n\t"                                                             \
      "addc.cc.u32 %4, %4, %13;\n\t"                                                             \
      "addc.cc.u32 %5, %5, %14;\n\t"                                                             \
      "addc.cc.u32 %6, %6, %15;\n\t"                                                             \
      "addc.cc.u32 %7, %7, %16;\n\t"                                                             \
      "addc.u32    %8, 0, 0;"                                                                     \
      : "+r"(t[i]), "+r"(t[i + 1]), "+r"(t[i + 2]), "+r"(t[i + 3]), "+r"(t[i + 4]), "+r"(t[i + 5]), \
        "+r"(t[i + 6]), "+r"(t[i + 7]), "=&r"(t[i + 8])                                           \
      : "r"((uint32_t)d[0]), "r"((uint32_t)d[1]), "r"((uint32_t)d[2]), "r"((uint32_t)d[3]),       \
        "r"((uint32_t)d[4]), "r"((uint32_t)d[5]), "r"((uint32_t)d[6]), "r"((uint32_t)d[7]))
#define ZKG_ADD_LO_ACC(t, i, d)                                                                  \
  asm("add.cc.u32  %0, %0, %9;\n\t"                                                              \
      "addc.cc.u32 %1, %1, %10;\n\t"                                                             \
      "addc.cc.u32 %2, %2, %11;\n\t"                                                             \
      "addc.cc.u32 %3, %3, %12;\n\t"                                                             \
      "addc.cc.u32 %4, %4, %13;\n\t"                                                             \
      "addc.cc.u32 %5, %5, %14;\n\t"                                                             \
      "addc.cc.u32 %6, %6, %15;\n\t"                                                             \
      "addc.cc.u32 %7, %7, %16;\n\t"                                                             \
      "addc.u32    %8, %8, 0;"                                                                    \
      : "+r"(t[i]), "+r"(t[i + 1]), "+r"(t[i + 2]), "+r"(t[i + 3]), "+r"(t[i + 4]), "+r"(t[i + 5]), \
        "+r"(t[i + 6]), "+r"(t[i + 7]), "+r"(t[i + 8])                                            \
      : "r"((uint32_t)d[0]), "r"((uint32_t)d[1]), "r"((uint32_t)d[2]), "r"((uint32_t)d[3]),       \
        "r"((uint32_t)d[4]), "r"((uint32_t)d[5]), "r"((uint32_t)d[6]), "r"((uint32_t)d[7]))
#define ZKG_ADD_HI(t, i, d)                                                                      \
  asm("add.cc.u32  %0, %0, %8;\n\t"                                                              \
      "addc.cc.u32 %1, %1, %9;\n\t"                                                              \
      "addc.cc.u32 %2, %2, %10;\n\t"                                                             \
      "addc.cc.u32 %3, %3, %11;\n\t"                                                             \
      "addc.cc.u32 %4, %4, %12;\n\t"                                                             \
      "addc.cc.u32 %5, %5, %13;\n\t"                                                             \
      "addc.cc.u32 %6, %6, %14;\n\t"                                                             \
      "addc.u32    %7, %7, %15;"                                                                  \
      : "+r"(t[i + 1]), "+r"(t[i + 2]), "+r"(t[i + 3]), "+r"(t[i + 4]), "+r"(t[i + 5]),           \
        "+r"(t[i + 6]), "+r"(t[i + 7]), "+r"(t[i + 8])                                            \
      : "r"((uint32_t)(d[0] >> 32)), "r"((uint32_t)(d[1] >> 32)), "r"((uint32_t)(d[2] >> 32)),    \
        "r"((uint32_t)(d[3] >> 32)), "r"((uint32_t)(d[4] >> 32)), "r"((uint32_t)(d[5] >> 32)),    \
        "r"((uint32_t)(d[6] >> 32)), "r"((uint32_t)(d[7] >> 32)))

// Mixed forms: one row kind with mad.wide + one chain, the other with mul.wide + two chains.
// PROD_WIDE selects the product rows' form (true: mad.wide), the reduction rows take the other.
template <class P, bool PROD_WIDE>
__device__ __forceinline__ Fp<P> mont_mul_mixed(const Fp<P>& a, const Fp<P>& b) {
  constexpr uint32_t q[8] = {P::P0, P::P1, P::P2, P::P3, P::P4, P::P5, P::P6, P::P7};
  uint32_t t[17];
#pragma unroll
  for (int i = 0; i < 8; i++) t[i] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    uint64_t d[8];
    if constexpr (PROD_WIDE) {
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = (uint64_t)a.w[j] * b.w[i] + t[i + j];
      t[i] = (uint32_t)d[0];
      ZKG_WIDE_CHAIN_FRESH(t, i, d);
    } else {
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = (uint64_t)a.w[j] * b.w[i];
      ZKG_ADD_LO_FRESH(t, i, d);
      ZKG_ADD_HI(t, i, d);
    }
    const uint32_t m = t[i] * P::INV;
    if constexpr (PROD_WIDE) {
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = (uint64_t)m * q[j];
      ZKG_ADD_LO_ACC(t, i, d);
      ZKG_ADD_HI(t, i, d);
    } else {
#pragma unroll
      for (int j = 0; j < 8; j++) d[j] = (uint64_t)m * q[j] + t[i + j];
      ZKG_WIDE_CHAIN_ACC(t, i, d);
    }
  }
  Fp<P> s, d;
#pragma unroll
  for (int i = 0; i < 8; i++) s.w[i] = t[8 + i];
  uint32_t borrow;
  asm("sub.cc.u32  %0, %9, %17;\n\t"
      "subc.cc.u32 %1, %10, %18;\n\t"
      "subc.cc.u32 %2, %11, %19;\n\t"
      "subc.cc.u32 %3, %12, %20;\n\t"
      "subc.cc.u32 %4, %13, %21;\n\t"
      "subc.cc.u32 %5, %14, %22;\n\t"
      "subc.cc.u32 %6, %15, %23;\n\t"
      "subc.cc.u32 %7, %16, %24;\n\t"
      "subc.u32    %8, 0, 0;"
      : "=&r"(d.w[0]), "=&r"(d.w[1]), "=&r"(d.w[2]), "=&r"(d.w[3]), "=&r"(d.w[4]), "=&r"(d.w[5]), "=&r"(d.w[6]),
        "=&r"(d.w[7]), "=&r"(borrow)
      : "r"(s.w[0]), "r"(s.w[1]), "r"(s.w[2]), "r"(s.w[3]), "r"(s.w[4]), "r"(s.w[5]), "r"(s.w[6]), "r"(s.w[7]),
        "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5), "n"(P::P6), "n"(P::P7));
  Fp<P> r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = (s.w[i] & borrow) | (d.w[i] & ~borrow);
  return r;
}

// The product the library uses: product rows as plain mul.wide with two add chains, reduction
// rows as mad.wide with one chain (measured 49.6 G products/s against 48.5 for mad.wide in both
// row kinds and 45.4 for mul.wide in both: the mix balances the multiply and add pipes).
template <class P>
__device__ __forceinline__ Fp<P> mont_mul_prod(const Fp<P>& a, const Fp<P>& b) {
  return mont_mul_mixed<P, false>(a, b);
}

template <class P>
__device__ __noinline__ Fp<P> mont_mul_call(Fp<P> a, Fp<P> b) {
  return mont_mul_prod(a, b);
}

template <class P>
__device__ __forceinline__ Fp<P> operator*(const Fp<P>& a, const Fp<P>& b) {
  if constexpr (P::kCompact) return mont_mul_call<P>(a, b);
  else return mont_mul_prod(a, b);
}

template <class P>
__device__ __forceinline__ Fp<P> sqr(const Fp<P>& a) {
  return a * a;
}

// Two independent products. In the compact form they share one out-of-line call, so the two
// dependency chains interleave (a lone thread, as in the window combination, otherwise waits
// on one product's chain at a time) and half the calls are made.
template <class P>
struct FpPair {
  Fp<P> x, y;
};

template <class P>
__device__ __noinline__ FpPair<P> mont_mul2_call(Fp<P> a, Fp<P> b, Fp<P> c, Fp<P> d) {
  return FpPair<P>{mont_mul_prod(a, b), mont_mul_prod(c, d)};
}

template <class P>
__device__ __forceinline__ void mul2(const Fp<P>& a, const Fp<P>& b, const Fp<P>& c, const Fp<P>& d, Fp<P>& r1,
                                     Fp<P>& r2) {
  if constexpr (P::kPairs) {
    FpPair<P> q = mont_mul2_call<P>(a, b, c, d);
    r1 = q.x;
    r2 = q.y;
  } else if constexpr (P::kCompact) {
    r1 = mont_mul_call<P>(a, b);
    r2 = mont_mul_call<P>(c, d);
  } else {
    r1 = mont_mul_prod(a, b);
    r2 = mont_mul_prod(c, d);
  }
}

// ------------------------------------------------------------------ memory helpers

// 32-byte element loads/stores as two 16-byte vector accesses (the address must be 16-byte
// aligned; every buffer and element offset in this library is).
template <class F>
__device__ __forceinline__ F load_fe(const void* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 lo = q[0], hi = q[1];
  F r;
  r.w[0] = lo.x; r.w[1] = lo.y; r.w[2] = lo.z; r.w[3] = lo.w;
  r.w[4] = hi.x; r.w[5] = hi.y; r.w[6] = hi.z; r.w[7] = hi.w;
  return r;
}

template <class F>
__device__ __forceinline__ F load_fe_cg(const void* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  uint4 lo = __ldcg(q), hi = __ldcg(q + 1);
  F r;
  r.w[0] = lo.x; r.w[1] = lo.y; r.w[2] = lo.z; r.w[3] = lo.w;
  r.w[4] = hi.x; r.w[5] = hi.y; r.w[6] = hi.z; r.w[7] = hi.w;
  return r;
}

template <class F>
__device__ __forceinline__ void store_fe(void* p, const F& a) {
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(a.w[0], a.w[1], a.w[2], a.w[3]);
  q[1] = make_uint4(a.w[4], a.w[5], a.w[6], a.w[7]);
}

// ------------------------------------------------------------------ Fq2 = Fq[u] / (u^2 + 1)

// a + b*u. Karatsuba product in three Fq products, square in two (the reference's G2 prelude,
// src/group.rs:38-48). B is the base field type (Fq, or its compact form FqC).
template <class B>
struct Fq2T {
  B a, b;
  __device__ __forceinline__ static Fq2T zero() { return Fq2T{B::zero(), B::zero()}; }
  __device__ __forceinline__ static Fq2T one() { return Fq2T{B::one(), B::zero()}; }
  __device__ __forceinline__ bool is_zero() const { return a.is_zero() && b.is_zero(); }
  __device__ __forceinline__ bool operator==(const Fq2T& o) const { return a == o.a && b == o.b; }
};

template <class B>
__device__ __forceinline__ Fq2T<B> operator+(const Fq2T<B>& x, const Fq2T<B>& y) {
  return Fq2T<B>{x.a + y.a, x.b + y.b};
}
template <class B>
__device__ __forceinline__ Fq2T<B> operator-(const Fq2T<B>& x, const Fq2T<B>& y) {
  return Fq2T<B>{x.a - y.a, x.b - y.b};
}
template <class B>
__device__ __forceinline__ Fq2T<B> neg(const Fq2T<B>& x) {
  return Fq2T<B>{neg(x.a), neg(x.b)};
}
template <class B>
__device__ __forceinline__ Fq2T<B> dbl(const Fq2T<B>& x) {
  return Fq2T<B>{x.a + x.a, x.b + x.b};
}
template <class B>
__device__ __forceinline__ Fq2T<B> operator*(const Fq2T<B>& x, const Fq2T<B>& y) {
  B ac = x.a * y.a;
  B bd = x.b * y.b;
  B cross = (x.a + x.b) * (y.a + y.b);
  return Fq2T<B>{ac - bd, (cross - ac) - bd};
}
template <class B>
__device__ __forceinline__ Fq2T<B> sqr(const Fq2T<B>& x) {
  B ab = x.a * x.b;
  return Fq2T<B>{(x.a + x.b) * (x.a - x.b), ab + ab};
}

// Two independent Fq2 products: the three Karatsuba base products of each, paired.
template <class B>
__device__ __forceinline__ void mul2(const Fq2T<B>& x, const Fq2T<B>& y, const Fq2T<B>& z, const Fq2T<B>& w,
                                     Fq2T<B>& r1, Fq2T<B>& r2) {
  B ac1, ac2, bd1, bd2, cr1, cr2;
  mul2(x.a, y.a, z.a, w.a, ac1, ac2);
  mul2(x.b, y.b, z.b, w.b, bd1, bd2);
  mul2(x.a + x.b, y.a + y.b, z.a + z.b, w.a + w.b, cr1, cr2);
  r1 = Fq2T<B>{ac1 - bd1, (cr1 - ac1) - bd1};
  r2 = Fq2T<B>{ac2 - bd2, (cr2 - ac2) - bd2};
}

// Two independent squarings. Fq: a pair of products (mul2). Fq2: (a+b)(a-b) and ab per element,
// two base products instead of three, paired across the two elements.
template <class P>
__device__ __forceinline__ void sqr2(const Fp<P>& x, const Fp<P>& y, Fp<P>& rx, Fp<P>& ry) {
  mul2(x, x, y, y, rx, ry);
}
template <class B>
__device__ __forceinline__ void sqr2(const Fq2T<B>& x, const Fq2T<B>& y, Fq2T<B>& rx, Fq2T<B>& ry) {
  B re_x, re_y, ab_x, ab_y;
  mul2(x.a + x.b, x.a - x.b, y.a + y.b, y.a - y.b, re_x, re_y);
  mul2(x.a, x.b, y.a, y.b, ab_x, ab_y);
  rx = Fq2T<B>{re_x, ab_x + ab_x};
  ry = Fq2T<B>{re_y, ab_y + ab_y};
}

using Fq2 = Fq2T<Fq>;
using Fq2C = Fq2T<FqC>;
using Fq2CP = Fq2T<FqCP>;

// The compact forms of a coordinate field (same memory layout): out-of-line products one at a
// time (CompactOf) or two at a time (PairedOf).
template <class F>
struct CompactOf;
template <>
struct CompactOf<Fq> {
  using type = FqC;
};
template <>
struct CompactOf<Fq2> {
  using type = Fq2C;
};
template <class F>
struct PairedOf;
template <>
struct PairedOf<Fq> {
  using type = FqCP;
};
template <>
struct PairedOf<Fq2> {
  using type = Fq2CP;
};

template <class F>
struct FieldWords;
template <>
struct FieldWords<Fq> {
  static constexpr int value = 8;
};
template <>
struct FieldWords<Fr> {
  static constexpr int value = 8;
};
template <>
struct FieldWords<FqC> {
  static constexpr int value = 8;
};
template <>
struct FieldWords<FqCP> {
  static constexpr int value = 8;
};
template <>
struct FieldWords<Fq2> {
  static constexpr int value = 16;
};
template <>
struct FieldWords<Fq2CP> {
  static constexpr int value = 16;
};
template <>
struct FieldWords<Fq2C> {
  static constexpr int value = 16;
};

template <class F>
__device__ __forceinline__ F load_elem(const uint32_t* p);
template <>
__device__ __forceinline__ Fq load_elem<Fq>(const uint32_t* p) {
  return load_fe<Fq>(p);
}
template <>
__device__ __forceinline__ Fr load_elem<Fr>(const uint32_t* p) {
  return load_fe<Fr>(p);
}
template <>
__device__ __forceinline__ FqC load_elem<FqC>(const uint32_t* p) {
  return load_fe<FqC>(p);
}
template <>
__device__ __forceinline__ FqCP load_elem<FqCP>(const uint32_t* p) {
  return load_fe<FqCP>(p);
}
template <>
__device__ __forceinline__ Fq2CP load_elem<Fq2CP>(const uint32_t* p) {
  return Fq2CP{load_fe<FqCP>(p), load_fe<FqCP>(p + 8)};
}
template <>
__device__ __forceinline__ Fq2 load_elem<Fq2>(const uint32_t* p) {
  return Fq2{load_fe<Fq>(p), load_fe<Fq>(p + 8)};
}
template <>
__device__ __forceinline__ Fq2C load_elem<Fq2C>(const uint32_t* p) {
  return Fq2C{load_fe<FqC>(p), load_fe<FqC>(p + 8)};
}

__device__ __forceinline__ void store_elem(uint32_t* p, const Fq& x) { store_fe(p, x); }
__device__ __forceinline__ void store_elem(uint32_t* p, const Fr& x) { store_fe(p, x); }
__device__ __forceinline__ void store_elem(uint32_t* p, const FqC& x) { store_fe(p, x); }
__device__ __forceinline__ void store_elem(uint32_t* p, const FqCP& x) { store_fe(p, x); }
template <class B>
__device__ __forceinline__ void store_elem(uint32_t* p, const Fq2T<B>& x) {
  store_fe(p, x.a);
  store_fe(p + 8, x.b);
}

}  // namespace zkg
