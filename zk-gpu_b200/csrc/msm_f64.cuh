// G1 bucket accumulation on the double-precision pipe (accumulation variants 3 and 4).
//
// Same segment walk as msm_accumulate (msm_kernels.cuh) and the same mixed addition
// (madd-2008-s), but the bucket sums are kept as five 52-bit limbs per coordinate in
// Montgomery form with R = 2^260 (field_f64.cuh), whose products issue on the FP64 pipe
// (measured on B200: 65 G Fq products/s against 50 G/s for the 32-bit integer product).
// Bases stay in the library's R = 2^256 word format: a canonical word value w becomes the
// limbs of 16 w, the same element in R = 2^260 form (unreduced, below 16p). Buckets and heads
// are written back as canonical R = 2^256 words, so the merge and reduction stages are the
// integer ones.
//
// Bounds (p < 2^254; a product of two values below 2^256 is below 2p):
//   bucket X, Y, ZZ, ZZZ < 2p;  base X2, Y2 < 16p;
//   U2 = X2 ZZ, S2 = Y2 ZZZ < 2p;  P = U2 - X + 2p, R = S2 - Y + 2p in (0, 4p);
//   PP, RR, PPP, Q < 2p;  D = 2Q < 4p;  X3 = RR + 6p - PPP - D in (0, 8p), reduced to [0, 2p);
//   V = Q - X3 + 2p < 4p;  Y3 = R V - Y PPP + 2p in (0, 4p), reduced to [0, 2p);
//   ZZ3 = ZZ PP, ZZZ3 = ZZZ PPP < 2p.
// P = 0 mod p (P is p, 2p or 3p) is the doubling / cancellation case; it is rare and runs the
// integer doubling on the canonical words.
#pragma once
#include "field_f64.cuh"
#include "msm_kernels.cuh"

namespace zkg {
namespace f64 {

__device__ const MultiplesOfP g_multiples_of_p = MultiplesOfP();

struct XyzzD {
  FqD x, y, zz, zzz;
};

struct Words8 {
  uint32_t w[8];
};

// Canonical R = 2^256 words of an R = 2^260 element below 2p (out of line: cold paths only).
static __device__ __noinline__ Words8 fqd_words_call(FqD a) {
  Words8 r;
  fqd_to_words(a, r.w);
  return r;
}

__device__ __forceinline__ void fqd_store_coord(uint32_t* p, const FqD& a, bool empty) {
  Words8 v;
  if (empty) {
#pragma unroll
    for (int i = 0; i < 8; i++) v.w[i] = 0;
  } else {
    v = fqd_words_call(a);
  }
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(v.w[0], v.w[1], v.w[2], v.w[3]);
  q[1] = make_uint4(v.w[4], v.w[5], v.w[6], v.w[7]);
}

// Canonical R = 2^256 words (x, y, zz, zzz), or all zeros for infinity.
__device__ __forceinline__ void fqd_store_xyzz(uint32_t* p, const XyzzD& a, bool empty) {
  fqd_store_coord(p, a.x, empty);
  fqd_store_coord(p + 8, a.y, empty);
  fqd_store_coord(p + 16, a.zz, empty);
  fqd_store_coord(p + 24, a.zzz, empty);
}

__device__ __forceinline__ FqD fqd_from_words(const FqC& a, const MultiplesOfP* kp) {
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w[i] = a.w[i];
  return fqd_reduce(fqd_from_words_x16(w), kp);
}

// 2 acc through the integer doubling (rare: equal points in one bucket). Every call passes
// at most 128 bytes of arguments, so the accumulator stays in registers. Returns false for
// infinity.
__device__ __forceinline__ bool xyzzd_double_slow(XyzzD& acc, const MultiplesOfP* kp) {
  Xyzz<FqC> p;
  const Words8 x = fqd_words_call(acc.x), y = fqd_words_call(acc.y);
  const Words8 zz = fqd_words_call(acc.zz), zzz = fqd_words_call(acc.zzz);
#pragma unroll
  for (int i = 0; i < 8; i++) {
    p.x.w[i] = x.w[i];
    p.y.w[i] = y.w[i];
    p.zz.w[i] = zz.w[i];
    p.zzz.w[i] = zzz.w[i];
  }
  const Xyzz<FqC> d = xyzz_double_call(p);
  if (d.zz.is_zero()) return false;
  acc = XyzzD{fqd_from_words(d.x, kp), fqd_from_words(d.y, kp), fqd_from_words(d.zz, kp), fqd_from_words(d.zzz, kp)};
  return true;
}

// acc += (bx, by) with acc not at infinity (madd-2008-s). Returns false when the sum is
// infinity.
template <bool PAIRS>
__device__ __forceinline__ bool xyzzd_add_affine(XyzzD& acc, const FqD& bx, const FqD& by,
                                                 const MultiplesOfP* kp) {
  FqD u2, s2;
  fqd_mul2<PAIRS>(bx, acc.zz, by, acc.zzz, u2, s2);
  const FqD pp = fqd_sub<2>(u2, acc.x);
  const FqD r = fqd_sub<2>(s2, acc.y);
  if (fqd_maybe_zero4(pp) && fqd_is_zero4(pp)) {
    if (!fqd_is_zero4(r)) return false;
    return xyzzd_double_slow(acc, kp);
  }
  FqD ppsq, rr, ppp, q;
  fqd_mul2<PAIRS>(pp, pp, r, r, ppsq, rr);
  fqd_mul2<PAIRS>(pp, ppsq, acc.x, ppsq, ppp, q);
  const FqD d = fqd_add(q, q);
  const FqD x3 = fqd_reduce(fqd_sub2<6>(rr, ppp, d), kp);
  const FqD v = fqd_sub<2>(q, x3);
  FqD t, yppp;
  fqd_mul2<PAIRS>(r, v, acc.y, ppp, t, yppp);
  const FqD y3 = fqd_reduce(fqd_sub<2>(t, yppp), kp);
  FqD zz3, zzz3;
  fqd_mul2<PAIRS>(acc.zz, ppsq, acc.zzz, ppp, zz3, zzz3);
  acc = XyzzD{x3, y3, zz3, zzz3};
  return true;
}

}  // namespace f64

// msm_accumulate (msm_kernels.cuh) for G1 with the bucket arithmetic in double-precision limbs;
// PAIRS: two products per out-of-line call, else one.
template <bool PAIRS>
__global__ void __launch_bounds__(128) msm_accumulate_f64(const uint32_t* __restrict__ bases,
                                                          const uint32_t* __restrict__ sorted,
                                                          const uint32_t* __restrict__ slot_start, uint32_t num_slots,
                                                          uint32_t seg_len, uint32_t* __restrict__ buckets,
                                                          uint32_t* __restrict__ heads,
                                                          uint32_t* __restrict__ head_keys) {
  using namespace f64;
  constexpr int XW = PointWords<Fq>::xyzz;
  const MultiplesOfP* kp = &g_multiples_of_p;
  const uint32_t total = __ldg(&slot_start[num_slots]);
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t p0_64 = (uint64_t)t * seg_len;
  if (p0_64 >= total) return;
  const uint32_t p0 = (uint32_t)p0_64;
  const uint64_t e64 = p0_64 + seg_len;
  const uint32_t p1 = e64 < total ? (uint32_t)e64 : total;

  uint32_t s = last_leq(slot_start, 0, num_slots, p0);
  uint32_t end = __ldg(&slot_start[s + 1]);
  bool head = __ldg(&slot_start[s]) < p0;
  uint32_t head_key = kNoKey;

  XyzzD acc;
  bool empty = true;
  uint32_t entry = __ldg(&sorted[p0]);
  Affine<Fq> next = load_signed_base<Fq>(bases, entry);
  for (uint32_t p = p0; p < p1; p++) {
    const Affine<Fq> cur = next;
    if (p + 1 < p1) {
      entry = __ldg(&sorted[p + 1]);
      next = load_signed_base<Fq>(bases, entry);
    }
    if (p == end) {
      if (head) {
        fqd_store_xyzz(heads + (size_t)t * XW, acc, empty);
        head_key = s;
        head = false;
      } else {
        fqd_store_xyzz(buckets + (size_t)s * XW, acc, empty);
      }
      empty = true;
      uint32_t s2 = s + 1;
      if (__ldg(&slot_start[s2 + 1]) <= p) s2 = last_leq(slot_start, s2, num_slots, p);
      s = s2;
      end = __ldg(&slot_start[s + 1]);
    }
    if (is_infinity(cur)) continue;
    uint32_t wx[8], wy[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      wx[i] = cur.x.w[i];
      wy[i] = cur.y.w[i];
    }
    const FqD bx = fqd_from_words_x16(wx), by = fqd_from_words_x16(wy);
    if (empty) {
      acc = XyzzD{fqd_reduce(bx, kp), fqd_reduce(by, kp), fqd_one260(), fqd_one260()};
      empty = false;
    } else {
      empty = !xyzzd_add_affine<PAIRS>(acc, bx, by, kp);
    }
  }
  if (head) {
    fqd_store_xyzz(heads + (size_t)t * XW, acc, empty);
    head_key = s;
  } else {
    fqd_store_xyzz(buckets + (size_t)s * XW, acc, empty);
  }
  head_keys[t] = head_key;
}

}  // namespace zkg
