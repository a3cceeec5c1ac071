// BN254 G1 (over Fq) and G2 (over Fq2) group law in XYZZ coordinates, device side.
//
// Restates src/shaders/curve.wgsl:1-96: x = X/ZZ, y = Y/ZZZ with ZZ^3 = ZZZ^2; infinity is
// ZZ = 0 (XYZZ) or (0, 0) (affine). Mixed addition madd-2008-s (8M + 2S), addition
// add-2008-s (12M + 2S), doubling dbl-2008-s-1 with a = 0 (6M + 3S), every special case
// (P = Q doubles, P = -Q gives infinity) handled exactly as the reference does.
#pragma once
#include "field.cuh"

namespace zkg {

template <class F>
struct Affine {
  F x, y;
};

template <class F>
struct Xyzz {
  F x, y, zz, zzz;
};

template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_infinity() {
  return Xyzz<F>{F::zero(), F::zero(), F::zero(), F::zero()};
}

template <class F>
__device__ __forceinline__ bool is_infinity(const Xyzz<F>& p) {
  return p.zz.is_zero();
}

template <class F>
__device__ __forceinline__ bool is_infinity(const Affine<F>& p) {
  return p.x.is_zero() && p.y.is_zero();
}

template <class F>
__device__ __forceinline__ Xyzz<F> from_affine(const Affine<F>& p) {
  if (is_infinity(p)) return xyzz_infinity<F>();
  return Xyzz<F>{p.x, p.y, F::one(), F::one()};
}

template <class F>
__device__ __forceinline__ Affine<F> negate(const Affine<F>& p) {
  return Affine<F>{p.x, neg(p.y)};
}

template <class F>
__device__ __forceinline__ Xyzz<F> negate(const Xyzz<F>& p) {
  return Xyzz<F>{p.x, neg(p.y), p.zz, p.zzz};
}

// 2P (dbl-2008-s-1, a = 0). Infinity stays infinity (ZZ = 0 gives ZZ3 = 0).
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_double(const Xyzz<F>& p) {
  F u = dbl(p.y);
  F v = sqr(u);
  F w = u * v;
  F s = p.x * v;
  F x2 = sqr(p.x);
  F m = dbl(x2) + x2;
  F x3 = sqr(m) - dbl(s);
  F y3 = m * (s - x3) - w * p.y;
  return Xyzz<F>{x3, y3, v * p.zz, w * p.zzz};
}

// The doubling branch of the additions (P = Q) is rare; keeping it out of line keeps the hot
// addition code small enough for the instruction cache.
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_double_call(Xyzz<F> p) {
  return xyzz_double(p);
}

// P + Q with Q affine (madd-2008-s).
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add_affine(const Xyzz<F>& p, const Affine<F>& q) {
  if (is_infinity(q)) return p;
  if (is_infinity(p)) return Xyzz<F>{q.x, q.y, F::one(), F::one()};
  F u2 = q.x * p.zz;
  F s2 = q.y * p.zzz;
  F pp = u2 - p.x;
  F r = s2 - p.y;
  if (pp.is_zero()) {
    if (r.is_zero()) return xyzz_double_call(p);
    return xyzz_infinity<F>();
  }
  F ppsq = sqr(pp);
  F ppp = pp * ppsq;
  F q_ = p.x * ppsq;
  F x3 = (sqr(r) - ppp) - dbl(q_);
  F y3 = r * (q_ - x3) - p.y * ppp;
  return Xyzz<F>{x3, y3, p.zz * ppsq, p.zzz * ppp};
}

// P + Q, both XYZZ (add-2008-s).
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add(const Xyzz<F>& p, const Xyzz<F>& q) {
  if (is_infinity(q)) return p;
  if (is_infinity(p)) return q;
  F u1 = p.x * q.zz;
  F u2 = q.x * p.zz;
  F s1 = p.y * q.zzz;
  F s2 = q.y * p.zzz;
  F pp = u2 - u1;
  F r = s2 - s1;
  if (pp.is_zero()) {
    if (r.is_zero()) return xyzz_double_call(p);
    return xyzz_infinity<F>();
  }
  F ppsq = sqr(pp);
  F ppp = pp * ppsq;
  F q_ = u1 * ppsq;
  F x3 = (sqr(r) - ppp) - dbl(q_);
  F y3 = r * (q_ - x3) - s1 * ppp;
  return Xyzz<F>{x3, y3, (p.zz * q.zz) * ppsq, (p.zzz * q.zzz) * ppp};
}

// ------------------------------------------------------------------ memory format
// Affine: x then y (FieldWords each); XYZZ: x, y, zz, zzz. Montgomery form, R = 2^256.

template <class F>
__device__ __forceinline__ Affine<F> load_affine(const uint32_t* p) {
  constexpr int W = FieldWords<F>::value;
  return Affine<F>{load_elem<F>(p), load_elem<F>(p + W)};
}

template <class F>
__device__ __forceinline__ Xyzz<F> load_xyzz(const uint32_t* p) {
  constexpr int W = FieldWords<F>::value;
  return Xyzz<F>{load_elem<F>(p), load_elem<F>(p + W), load_elem<F>(p + 2 * W), load_elem<F>(p + 3 * W)};
}

template <class F>
__device__ __forceinline__ void store_xyzz(uint32_t* p, const Xyzz<F>& a) {
  constexpr int W = FieldWords<F>::value;
  store_elem(p, a.x);
  store_elem(p + W, a.y);
  store_elem(p + 2 * W, a.zz);
  store_elem(p + 3 * W, a.zzz);
}

}  // namespace zkg
