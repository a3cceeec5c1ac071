// Montgomery products on the double-precision pipe: five 52-bit limbs held in doubles,
// R = 2^260.
//
// A 52 x 52-bit limb product a*b (< 2^104) is split exactly with two FMAs:
//   h = fma_rz(a, b, 2^104)            = 2^104 + floor(ab / 2^52) * 2^52   (ulp 2^52, truncated)
//   l = fma(a, b, (2^104 + 2^52) - h)  = 2^52 + (ab mod 2^52)              (exact: 2^52 <= l < 2^53)
// The bit patterns of h and l are the high and low halves plus a constant (the exponent field),
// so column sums are formed with 64-bit integer adds of the raw patterns and the constants are
// removed once per column (wrap-around arithmetic makes the intermediate overflow harmless).
// Every other double operation here is exact (integers below 2^53, or differences of multiples
// of 2^52 below 2^104), so only the high-half FMA depends on the rounding mode.
//
// Reduction: five digit steps in base 2^52, q_i = (t_i mod 2^52) * (-p^-1) mod 2^52; the low half
// of q_i * p_0 is never formed because t_i + lo(q_i p_0) is the next multiple of 2^52 at or
// above t_i, so the carry into column i+1 is ceil(t_i / 2^52). Inputs whose product is below
// p 2^260 (any two below 2^256) give an output below 2p (p < 2^254, R = 2^260).
#pragma once
#include <cstdint>

namespace zkg {
namespace f64 {

constexpr double kC104 = 20282409603651670423947251286016.0;  // 2^104
constexpr double kC52 = 4503599627370496.0;                   // 2^52
constexpr double kC104p52 = kC104 + kC52;                     // exact in a double
constexpr uint64_t kB104 = 0x4670000000000000ull;             // bit pattern of 2^104
constexpr uint64_t kB52 = 0x4330000000000000ull;              // bit pattern of 2^52
constexpr uint64_t kM52 = (1ull << 52) - 1;

struct FqLimbs {
  __host__ __device__ static constexpr uint64_t P(int j) {
    return j == 0 ? 0x8c16d87cfd47ull
         : j == 1 ? 0x916871ca8d3c2ull
         : j == 2 ? 0x181585d97816aull
         : j == 3 ? 0xa029b85045b68ull
                  : 0x30644e72e131ull;
  }
  static constexpr uint64_t PINV = 0x20782e4866389ull;  // -p^-1 mod 2^52
};
struct FrLimbs {
  __host__ __device__ static constexpr uint64_t P(int j) {
    return j == 0 ? 0x1f593f0000001ull
         : j == 1 ? 0x4879b9709143eull
         : j == 2 ? 0x181585d2833e8ull
         : j == 3 ? 0xa029b85045b68ull
                  : 0x30644e72e131ull;
  }
  static constexpr uint64_t PINV = 0x1f593efffffffull;
};

// Number of low-half (kB52) and high-half (kB104) patterns that a column receives.
constexpr int lo_terms(int k) {
  int n = 0;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      if (i + j == k) n++;          // product a_i b_j
      if (j >= 1 && i + j == k) n++;  // reduction q_i p_j, j >= 1
    }
  return n;
}
constexpr int hi_terms(int k) {
  int n = 0;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      if (i + j + 1 == k) n++;  // product
      if (i + j + 1 == k) n++;  // reduction (j = 0 contributes its high half only)
    }
  return n;
}
constexpr uint64_t column_bias(int k) { return (uint64_t)lo_terms(k) * kB52 + (uint64_t)hi_terms(k) * kB104; }

__device__ __forceinline__ uint64_t bits(double d) { return (uint64_t)__double_as_longlong(d); }
__device__ __forceinline__ double limb_to_double(uint64_t v) {  // v < 2^52
  return __dsub_rn(__longlong_as_double((long long)(v | kB52)), kC52);
}
__device__ __forceinline__ uint64_t double_to_limb(double d) {  // d an integer in [0, 2^52)
  return bits(__dadd_rn(d, kC52)) & kM52;
}

template <typename L>
__device__ __forceinline__ void mont_mul(const double (&x)[5], const double (&y)[5], double (&out)[5]) {
  uint64_t c[10];
#pragma unroll
  for (int k = 0; k < 10; k++) c[k] = 0ull - column_bias(k);
#pragma unroll
  for (int i = 0; i < 5; i++) {
#pragma unroll
    for (int j = 0; j < 5; j++) {
      double h = __fma_rz(x[i], y[j], kC104);
      double l = __fma_rn(x[i], y[j], __dsub_rn(kC104p52, h));
      c[i + j] += bits(l);
      c[i + j + 1] += bits(h);
    }
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const uint64_t t = c[i];
    // t + lo(q p_0) is the next multiple of 2^52 at or above t: carry = ceil(t / 2^52)
    const uint64_t carry = (t + kM52) >> 52;
    const double tf = limb_to_double(t & kM52);
    const double qh = __fma_rz(tf, (double)L::PINV, kC104);
    const double ql = __fma_rn(tf, (double)L::PINV, __dsub_rn(kC104p52, qh));
    const double q = __dsub_rn(ql, kC52);
    c[i + 1] += bits(__fma_rz(q, (double)L::P(0), kC104)) + carry;
#pragma unroll
    for (int j = 1; j < 5; j++) {
      double h = __fma_rz(q, (double)L::P(j), kC104);
      double l = __fma_rn(q, (double)L::P(j), __dsub_rn(kC104p52, h));
      c[i + j] += bits(l);
      c[i + j + 1] += bits(h);
    }
  }
  uint64_t carry = 0;
#pragma unroll
  for (int k = 5; k < 10; k++) {
    const uint64_t v = c[k] + carry;
    carry = v >> 52;
    out[k - 5] = limb_to_double(k < 9 ? (v & kM52) : v);
  }
}

// Bias of the reduction phase's patterns in column k (the product phase of mont_mul_sub adds
// and subtracts equal numbers of patterns, whose biases cancel).
constexpr int red_lo_terms(int k) {
  int n = 0;
  for (int i = 0; i < 5; i++)
    for (int j = 1; j < 5; j++)
      if (i + j == k) n++;
  return n;
}
constexpr int red_hi_terms(int k) {
  int n = 0;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++)
      if (i + j + 1 == k) n++;
  return n;
}
constexpr uint64_t red_bias(int k) { return (uint64_t)red_lo_terms(k) * kB52 + (uint64_t)red_hi_terms(k) * kB104; }

// Column k (base 2^52) of m 2^256, a multiple of m that is at least c d whenever c, d < 2m:
// m 2^256 = (m << 48) 2^208, so columns 4..9 hold the limbs of m << 48.
template <class L>
__host__ __device__ constexpr uint64_t shifted_modulus_limb(int k) {
  if (k < 4) return 0;
  const int j = k - 4;
  const uint64_t lo = j >= 1 ? (L::P(j - 1) >> 4) : 0;            // top 48 bits of limb j-1 -> bits 0..47
  const uint64_t hi = j < 5 ? ((L::P(j) & 0xfull) << 48) : 0;    // low 4 bits of limb j -> bits 48..51
  return lo | hi;
}

// (a b - c d + m 2^256) 2^-260 mod m in one Montgomery reduction: a, b below 4m and c, d below
// 2m give a result below 1.3m. The columns are signed (the difference of the two products can
// be negative in any column): carries are ceil(t / 2^52) by arithmetic shifts, and t mod 2^52
// is the two's complement residue.
template <typename L>
__device__ __forceinline__ void mont_mul_sub(const double (&a)[5], const double (&b)[5], const double (&c)[5],
                                             const double (&d)[5], double (&out)[5]) {
  int64_t col[10];
#pragma unroll
  for (int k = 0; k < 10; k++) col[k] = (int64_t)(shifted_modulus_limb<L>(k) - red_bias(k));
#pragma unroll
  for (int i = 0; i < 5; i++) {
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const double h = __fma_rz(a[i], b[j], kC104);
      const double l = __fma_rn(a[i], b[j], __dsub_rn(kC104p52, h));
      const double h2 = __fma_rz(c[i], d[j], kC104);
      const double l2 = __fma_rn(c[i], d[j], __dsub_rn(kC104p52, h2));
      col[i + j] += (int64_t)(bits(l) - bits(l2));
      col[i + j + 1] += (int64_t)(bits(h) - bits(h2));
    }
  }
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const int64_t t = col[i];
    const int64_t carry = (t + (int64_t)kM52) >> 52;  // ceil(t / 2^52), arithmetic shift
    const double tf = limb_to_double((uint64_t)t & kM52);
    const double qh = __fma_rz(tf, (double)L::PINV, kC104);
    const double ql = __fma_rn(tf, (double)L::PINV, __dsub_rn(kC104p52, qh));
    const double q = __dsub_rn(ql, kC52);
    col[i + 1] += (int64_t)bits(__fma_rz(q, (double)L::P(0), kC104)) + carry;
#pragma unroll
    for (int j = 1; j < 5; j++) {
      const double h = __fma_rz(q, (double)L::P(j), kC104);
      const double l = __fma_rn(q, (double)L::P(j), __dsub_rn(kC104p52, h));
      col[i + j] += (int64_t)bits(l);
      col[i + j + 1] += (int64_t)bits(h);
    }
  }
  int64_t carry = 0;
#pragma unroll
  for (int k = 5; k < 10; k++) {
    const int64_t v = col[k] + carry;
    carry = v >> 52;
    out[k - 5] = limb_to_double(k < 9 ? ((uint64_t)v & kM52) : (uint64_t)v);
  }
}

// 8 x 32-bit words (an integer below 2^255) <-> five 52-bit limbs.
__device__ __forceinline__ void words_to_limbs(const uint32_t (&w)[8], double (&out)[5]) {
  const uint64_t w0 = w[0] | (uint64_t)w[1] << 32, w1 = w[2] | (uint64_t)w[3] << 32;
  const uint64_t w2 = w[4] | (uint64_t)w[5] << 32, w3 = w[6] | (uint64_t)w[7] << 32;
  out[0] = limb_to_double(w0 & kM52);
  out[1] = limb_to_double(((w0 >> 52) | (w1 << 12)) & kM52);
  out[2] = limb_to_double(((w1 >> 40) | (w2 << 24)) & kM52);
  out[3] = limb_to_double(((w2 >> 28) | (w3 << 36)) & kM52);
  out[4] = limb_to_double(w3 >> 16);
}

__device__ __forceinline__ void limbs_to_words(const double (&x)[5], uint32_t (&w)[8]) {
  const uint64_t l0 = double_to_limb(x[0]), l1 = double_to_limb(x[1]), l2 = double_to_limb(x[2]);
  const uint64_t l3 = double_to_limb(x[3]), l4 = double_to_limb(x[4]);
  const uint64_t w0 = l0 | (l1 << 52), w1 = (l1 >> 12) | (l2 << 40), w2 = (l2 >> 24) | (l3 << 28);
  const uint64_t w3 = (l3 >> 36) | (l4 << 16);
  w[0] = (uint32_t)w0;
  w[1] = (uint32_t)(w0 >> 32);
  w[2] = (uint32_t)w1;
  w[3] = (uint32_t)(w1 >> 32);
  w[4] = (uint32_t)w2;
  w[5] = (uint32_t)(w2 >> 32);
  w[6] = (uint32_t)w3;
  w[7] = (uint32_t)(w3 >> 32);
}

// ------------------------------------------------------------------ Fq elements as limbs

// A field element (Fq, or Fr with the FrLimbs constants) as five normalized limbs (each an
// integer in [0, 2^52) held in a double), in Montgomery form with R = 2^260. The value is kept
// below a known small multiple of the modulus m (stated at every use); mont_mul keeps products
// below 2m for any inputs below 2^256.
struct FqD {
  double l[5];
};
struct FqDPair {
  FqD x, y;
};

// k*m in normalized limbs (compile time).
struct Limbs5 {
  uint64_t v[5];
};
template <class L = FqLimbs>
constexpr Limbs5 times_p(uint64_t k) {
  Limbs5 r{};
  uint64_t carry = 0;
  for (int j = 0; j < 5; j++) {
    const uint64_t t = k * L::P(j) + carry;
    r.v[j] = j < 4 ? (t & kM52) : t;
    carry = t >> 52;
  }
  return r;
}
template <class L = FqLimbs>
struct MultiplesOf {
  double v[16][5];
  constexpr MultiplesOf() : v() {
    for (int k = 0; k < 16; k++)
      for (int j = 0; j < 5; j++) v[k][j] = (double)times_p<L>((uint64_t)k).v[j];
  }
};
using MultiplesOfP = MultiplesOf<FqLimbs>;

constexpr double kFloorMagic = 6755399441055744.0;     // 1.5 * 2^52: fma_rd(t, s, M) - M = floor(t s)
constexpr double kInv2p52 = 1.0 / 4503599627370496.0;   // 2^-52
// <= 1 / (floor(m / 2^208) + 1); p and r share their top 46 bits, so one constant serves both.
constexpr double kInvP4 = 1.879438846411752e-14;

// 2^256 mod p and 2^260 mod p in limbs: multiplying by the first maps R = 2^260 Montgomery form
// to R = 2^256 form; the second is one in R = 2^260 form.
__device__ __forceinline__ FqD fqd_one256() {
  return FqD{{(double)0xd438dc58f0d9dull, (double)0x28f5c70b3dd35ull, (double)0x879462c0a78ebull,
              (double)0xdf2f666ea36f7ull, (double)0xe0a77c19a07ull}};
}
// One in R = 2^260 Montgomery form for Fr (2^260 mod r), the NTT's unit twiddle.
__device__ __forceinline__ FqD frd_one260() {
  return FqD{{(double)0xb6b753fffffacull, (double)0x380f271055b9dull, (double)0x18f016ecef7c8ull,
              (double)0x724f85a9201d8ull, (double)0x1f16424e1bb7ull}};
}
__device__ __forceinline__ FqD fqd_one260() {
  return FqD{{(double)0x20880f6fce4b4ull, (double)0x49baa989a8455ull, (double)0x18f014a498908ull,
              (double)0x724f85a9201d8ull, (double)0x1f16424e1bb7ull}};
}

template <int K, class L = FqLimbs>
__device__ __forceinline__ double kp_limb(int j) {
  return (double)times_p<L>(K).v[j];
}

// Signed carry propagation: limbwise values in (-2^53, 2^53) (exact integers) whose total is
// non-negative and below 2^260 become normalized limbs. floor(t / 2^52) comes from rounding
// t * 2^-52 + 1.5 * 2^52 toward minus infinity.
__device__ __forceinline__ FqD fqd_normalize(double t0, double t1, double t2, double t3, double t4) {
  double c;
  c = __dsub_rn(__fma_rd(t0, kInv2p52, kFloorMagic), kFloorMagic);
  t0 = __fma_rn(c, -kC52, t0);
  t1 = __dadd_rn(t1, c);
  c = __dsub_rn(__fma_rd(t1, kInv2p52, kFloorMagic), kFloorMagic);
  t1 = __fma_rn(c, -kC52, t1);
  t2 = __dadd_rn(t2, c);
  c = __dsub_rn(__fma_rd(t2, kInv2p52, kFloorMagic), kFloorMagic);
  t2 = __fma_rn(c, -kC52, t2);
  t3 = __dadd_rn(t3, c);
  c = __dsub_rn(__fma_rd(t3, kInv2p52, kFloorMagic), kFloorMagic);
  t3 = __fma_rn(c, -kC52, t3);
  t4 = __dadd_rn(t4, c);
  return FqD{{t0, t1, t2, t3, t4}};
}

// a - b + K m (K m >= b keeps the result positive; the result is below a + K m).
template <int K, class L = FqLimbs>
__device__ __forceinline__ FqD fqd_sub(const FqD& a, const FqD& b) {
  double t[5];
#pragma unroll
  for (int j = 0; j < 5; j++) t[j] = __dadd_rn(__dsub_rn(a.l[j], b.l[j]), kp_limb<K, L>(j));
  return fqd_normalize(t[0], t[1], t[2], t[3], t[4]);
}

__device__ __forceinline__ FqD fqd_add(const FqD& a, const FqD& b) {
  double t[5];
#pragma unroll
  for (int j = 0; j < 5; j++) t[j] = __dadd_rn(a.l[j], b.l[j]);
  return fqd_normalize(t[0], t[1], t[2], t[3], t[4]);
}

// a + K m - b - c (each operand normalized; K m >= b + c).
template <int K, class L = FqLimbs>
__device__ __forceinline__ FqD fqd_sub2(const FqD& a, const FqD& b, const FqD& c) {
  double t[5];
#pragma unroll
  for (int j = 0; j < 5; j++)
    t[j] = __dsub_rn(__dadd_rn(a.l[j], kp_limb<K, L>(j)), __dadd_rn(b.l[j], c.l[j]));
  return fqd_normalize(t[0], t[1], t[2], t[3], t[4]);
}

// x (below 16m) -> x - q m in [0, 2m), q from the top limb (q never exceeds floor(x / m), and
// falls short of it by at most one). kp holds k m, k = 0..15, in normalized limbs.
template <class L = FqLimbs>
__device__ __forceinline__ FqD fqd_reduce(const FqD& x, const MultiplesOf<L>* __restrict__ kp) {
  const double qm = __fma_rd(x.l[4], kInvP4, kFloorMagic);
  const int q = (int)((uint64_t)__double_as_longlong(qm) - (uint64_t)__double_as_longlong(kFloorMagic));
  const double* m = kp->v[q];
  double t[5];
#pragma unroll
  for (int j = 0; j < 5; j++) t[j] = __dsub_rn(x.l[j], __ldg(m + j));
  return fqd_normalize(t[0], t[1], t[2], t[3], t[4]);
}

// The product of two elements below 2^256 (result below 2m).
template <class L = FqLimbs>
__device__ __forceinline__ FqD fqd_mul(const FqD& a, const FqD& b) {
  FqD r;
  mont_mul<L>(a.l, b.l, r.l);
  return r;
}

// Two independent products per out-of-line call: the accumulation loop stays small enough for
// the instruction cache and each call carries two independent dependency chains.
template <class L = FqLimbs>
static __device__ __noinline__ FqDPair fqd_mul2_call(FqD a, FqD b, FqD c, FqD d) {
  return FqDPair{fqd_mul<L>(a, b), fqd_mul<L>(c, d)};
}

// a b - c d (Montgomery form, below 1.3m) for a, b below 4m and c, d below 2m, one call.
template <class L = FqLimbs>
static __device__ __noinline__ FqD fqd_mul_sub_call(FqD a, FqD b, FqD c, FqD d) {
  FqD r;
  mont_mul_sub<L>(a.l, b.l, c.l, d.l, r.l);
  return r;
}

// One product per out-of-line call.
template <class L = FqLimbs>
static __device__ __noinline__ FqD fqd_mul_call(FqD a, FqD b) {
  return fqd_mul<L>(a, b);
}

// Two independent products: one call for both (PAIRS) or one call each.
template <bool PAIRS, class L = FqLimbs>
__device__ __forceinline__ void fqd_mul2(const FqD& a, const FqD& b, const FqD& c, const FqD& d, FqD& r1,
                                         FqD& r2) {
  if (PAIRS) {
    FqDPair q = fqd_mul2_call<L>(a, b, c, d);
    r1 = q.x;
    r2 = q.y;
  } else {
    r1 = fqd_mul_call<L>(a, b);
    r2 = fqd_mul_call<L>(c, d);
  }
}

// Low-limb filter for x == k p, k = 1..3 (x below 4p): exact test follows only when it passes.
__device__ __forceinline__ bool fqd_maybe_zero4(const FqD& x) {
  return x.l[0] == kp_limb<1>(0) || x.l[0] == kp_limb<2>(0) || x.l[0] == kp_limb<3>(0);
}
// x (below 4p) is 0 mod p: x is p, 2p or 3p (x > 0 where this is used).
__device__ __forceinline__ bool fqd_is_zero4(const FqD& x) {
  bool e1 = true, e2 = true, e3 = true;
#pragma unroll
  for (int j = 0; j < 5; j++) {
    e1 = e1 && x.l[j] == kp_limb<1>(j);
    e2 = e2 && x.l[j] == kp_limb<2>(j);
    e3 = e3 && x.l[j] == kp_limb<3>(j);
  }
  return e1 || e2 || e3;
}

// 16 w for an integer w < 2^256 held as 8 words (the top limb may reach 2^52 - 1): converts a
// canonical R = 2^256 Montgomery value into an (unreduced, below 16p) R = 2^260 one.
__device__ __forceinline__ FqD fqd_from_words_x16(const uint32_t (&w)[8]) {
  const uint64_t w0 = w[0] | (uint64_t)w[1] << 32, w1 = w[2] | (uint64_t)w[3] << 32;
  const uint64_t w2 = w[4] | (uint64_t)w[5] << 32, w3 = w[6] | (uint64_t)w[7] << 32;
  return FqD{{limb_to_double((w0 << 4) & kM52), limb_to_double(((w0 >> 48) | (w1 << 16)) & kM52),
              limb_to_double(((w1 >> 36) | (w2 << 28)) & kM52), limb_to_double(((w2 >> 24) | (w3 << 40)) & kM52),
              limb_to_double(w3 >> 12)}};
}

// An R = 2^260 element below 2p -> canonical R = 2^256 words.
__device__ __forceinline__ void fqd_to_words(const FqD& x, uint32_t (&w)[8]) {
  FqD y = fqd_mul(x, fqd_one256());  // below 2p
  limbs_to_words(y.l, w);
  // subtract p when w >= p
  const uint32_t pw[8] = {0xd87cfd47u, 0x3c208c16u, 0x6871ca8du, 0x97816a91u,
                          0x8181585du, 0xb85045b6u, 0xe131a029u, 0x30644e72u};
  uint32_t d[8];
  uint32_t borrow = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint64_t t = (uint64_t)w[i] - pw[i] - borrow;
    d[i] = (uint32_t)t;
    borrow = (uint32_t)(t >> 63);
  }
  if (!borrow) {
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = d[i];
  }
}

}  // namespace f64
}  // namespace zkg
