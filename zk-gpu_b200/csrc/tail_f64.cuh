// Fq on the double-precision pipe for the G1 MSM's tail stages (merge levels, running-sum
// reductions, window sums, Horner combination): FqT plugs into the generic XYZZ formulas of
// curve.cuh and the lane-parallel ones of curve_lanes.cuh, in place of the 32-bit integer pairs.
//
// The tails are dependent chains of point additions run by few threads (a 2^16 MSM's reduction
// has one block per window, its combination one warp), so the latency of one field product sets
// their time. The integer Montgomery product is a chain of carry-propagating multiply-adds row
// after row; the limb product (field_f64.cuh) forms its 25 partial products independently and
// only its five reduction steps depend on each other.
//
// Every FqT value stays below 2p (R = 2^260 Montgomery form): sums and differences are reduced
// back below 2p at once (fqd_reduce), products of two values below 2p are below 2p. Memory
// holds the library's canonical R = 2^256 words: loads scale by 16 and reduce, stores multiply by
// 2^256 / 2^260 and subtract p when needed (fqd_to_words).
#pragma once
#include "msm_f64.cuh"

namespace zkg {

struct FqT {
  f64::FqD v;
  __device__ __forceinline__ static FqT zero() { return FqT{{{0.0, 0.0, 0.0, 0.0, 0.0}}}; }
  __device__ __forceinline__ static FqT one() { return FqT{f64::fqd_one260()}; }
  // 0 or p (the values below 2p congruent to 0)
  __device__ __forceinline__ bool is_zero() const {
    bool z = true, p = true;
#pragma unroll
    for (int j = 0; j < 5; j++) {
      z = z && v.l[j] == 0.0;
      p = p && v.l[j] == f64::kp_limb<1>(j);
    }
    return z || p;
  }
};

__device__ __forceinline__ FqT fqt_reduce(const f64::FqD& x) {  // x below 16p
  return FqT{f64::fqd_reduce(x, &f64::g_multiples_of_p)};
}
__device__ __forceinline__ FqT operator+(const FqT& a, const FqT& b) { return fqt_reduce(f64::fqd_add(a.v, b.v)); }
__device__ __forceinline__ FqT operator-(const FqT& a, const FqT& b) {  // a - b + 2p in (0, 4p)
  return fqt_reduce(f64::fqd_sub<2>(a.v, b.v));
}
__device__ __forceinline__ FqT dbl(const FqT& a) { return a + a; }
__device__ __forceinline__ FqT neg(const FqT& a) { return FqT::zero() - a; }
// One product per out-of-line call (the tail kernels' code stays small).
__device__ __forceinline__ FqT operator*(const FqT& a, const FqT& b) { return FqT{f64::fqd_mul_call(a.v, b.v)}; }
// Two independent products in one call: their reduction chains interleave.
__device__ __forceinline__ void mul2(const FqT& a, const FqT& b, const FqT& c, const FqT& d, FqT& r1, FqT& r2) {
  const f64::FqDPair q = f64::fqd_mul2_call(a.v, b.v, c.v, d.v);
  r1 = FqT{q.x};
  r2 = FqT{q.y};
}
__device__ __forceinline__ void sqr2(const FqT& x, const FqT& y, FqT& rx, FqT& ry) { mul2(x, x, y, y, rx, ry); }

template <>
struct FieldWords<FqT> {
  static constexpr int value = 8;
};
template <>
__device__ __forceinline__ FqT load_elem<FqT>(const uint32_t* p) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
  const uint4 lo = q[0], hi = q[1];
  const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
  return fqt_reduce(f64::fqd_from_words_x16(w));
}
__device__ __forceinline__ void store_elem(uint32_t* p, const FqT& a) {
  uint32_t w[8];
  f64::fqd_to_words(a.v, w);
  uint4* q = reinterpret_cast<uint4*>(p);
  q[0] = make_uint4(w[0], w[1], w[2], w[3]);
  q[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// Lane exchange for curve_lanes.cuh: five doubles per lane.
template <>
struct LaneWords<FqT> {
  static constexpr int value = 10;
};
__device__ __forceinline__ void lane_put(LaneScratch sm, const FqT& v) {
  double* d = reinterpret_cast<double*>(sm.words) + 5 * (threadIdx.x & 31);
#pragma unroll
  for (int i = 0; i < 5; i++) d[i] = v.v.l[i];
}
__device__ __forceinline__ FqT lane_get_t(LaneScratch sm, unsigned lane) {
  const double* d = reinterpret_cast<const double*>(sm.words) + 5 * lane;
  FqT v;
#pragma unroll
  for (int i = 0; i < 5; i++) v.v.l[i] = d[i];
  return v;
}
template <int K>
__device__ __forceinline__ void lane_mul(const FqT (&a)[K], const FqT (&b)[K], FqT (&r)[K], LaneScratch sm) {
  static_assert(K <= 32, "one product per lane");
  const unsigned lane = threadIdx.x & 31;
  FqT x = a[0], y = b[0];
#pragma unroll
  for (int k = 1; k < K; k++) {
    if (lane == (unsigned)k) {
      x = a[k];
      y = b[k];
    }
  }
  const FqT p = x * y;
  __syncwarp();
  lane_put(sm, p);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; k++) r[k] = lane_get_t(sm, k);
}

}  // namespace zkg
