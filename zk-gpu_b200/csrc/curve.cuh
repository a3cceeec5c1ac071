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

// 2P (dbl-2008-s-1, a = 0). Infinity stays infinity (ZZ = 0 gives ZZ3 = 0). The nine
// products go in five steps of independent pairs.
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_double(const Xyzz<F>& p) {
  F u = dbl(p.y);
  F v, x2, w, s, m2, wy, zz3, zzz3;
  sqr2(u, p.x, v, x2);
  mul2(u, v, p.x, v, w, s);
  F m = dbl(x2) + x2;
  mul2(m, m, w, p.y, m2, wy);
  F x3 = m2 - dbl(s);
  mul2(v, p.zz, w, p.zzz, zz3, zzz3);
  F y3 = m * (s - x3) - wy;
  return Xyzz<F>{x3, y3, zz3, zzz3};
}

// The doubling branch of the additions (P = Q) is rare; keeping it out of line keeps the hot
// addition code small enough for the instruction cache.
template <class F>
__device__ __noinline__ Xyzz<F> xyzz_double_call(Xyzz<F> p) {
  return xyzz_double(p);
}

// P + Q with Q affine (madd-2008-s): ten products in five pairs.
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add_affine(const Xyzz<F>& p, const Affine<F>& q) {
  if (is_infinity(q)) return p;
  if (is_infinity(p)) return Xyzz<F>{q.x, q.y, F::one(), F::one()};
  F u2, s2;
  mul2(q.x, p.zz, q.y, p.zzz, u2, s2);
  F pp = u2 - p.x;
  F r = s2 - p.y;
  if (pp.is_zero()) {
    if (r.is_zero()) return xyzz_double_call(p);
    return xyzz_infinity<F>();
  }
  F ppsq, rr, ppp, q_, zz3, zzz3, t, yppp;
  sqr2(pp, r, ppsq, rr);
  mul2(pp, ppsq, p.x, ppsq, ppp, q_);
  F x3 = (rr - ppp) - dbl(q_);
  mul2(r, q_ - x3, p.y, ppp, t, yppp);
  mul2(p.zz, ppsq, p.zzz, ppp, zz3, zzz3);
  return Xyzz<F>{x3, t - yppp, zz3, zzz3};
}

// P + Q, both XYZZ (add-2008-s): fourteen products in seven pairs.
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add(const Xyzz<F>& p, const Xyzz<F>& q) {
  if (is_infinity(q)) return p;
  if (is_infinity(p)) return q;
  F u1, u2, s1, s2;
  mul2(p.x, q.zz, q.x, p.zz, u1, u2);
  mul2(p.y, q.zzz, q.y, p.zzz, s1, s2);
  F pp = u2 - u1;
  F r = s2 - s1;
  if (pp.is_zero()) {
    if (r.is_zero()) return xyzz_double_call(p);
    return xyzz_infinity<F>();
  }
  F ppsq, rr, ppp, q_, zz12, zzz12, t, sppp, zz3, zzz3;
  sqr2(pp, r, ppsq, rr);
  mul2(pp, ppsq, u1, ppsq, ppp, q_);
  mul2(p.zz, q.zz, p.zzz, q.zzz, zz12, zzz12);
  F x3 = (rr - ppp) - dbl(q_);
  mul2(r, q_ - x3, s1, ppp, t, sppp);
  mul2(zz12, ppsq, zzz12, ppp, zz3, zzz3);
  return Xyzz<F>{x3, t - sppp, zz3, zzz3};
}

// ------------------------------------------------------------------ inversion (Fermat)

// a^(p-2) mod p, square-and-multiply over the exponent bits from the top (a != 0).
template <class P>
__device__ Fp<P> fp_inverse(const Fp<P>& a) {
  const uint32_t e[8] = {P::P0 - 2u, P::P1, P::P2, P::P3, P::P4, P::P5, P::P6, P::P7};  // p0 >= 2
  Fp<P> acc = Fp<P>::one();
  for (int bit = 255; bit >= 0; bit--) {
    acc = acc * acc;
    if ((e[bit >> 5] >> (bit & 31)) & 1) acc = acc * a;
  }
  return acc;
}

static __device__ Fq field_inverse(const Fq& a) { return fp_inverse(a); }
// 1 / (a + bu) = (a - bu) / (a^2 + b^2)
static __device__ Fq2 field_inverse(const Fq2& x) {
  Fq inv = fp_inverse(x.a * x.a + x.b * x.b);
  return Fq2{x.a * inv, neg(x.b * inv)};
}

// XYZZ -> affine with one inversion: I = 1/(ZZ*ZZZ), 1/ZZ = ZZZ*I, 1/ZZZ = ZZ*I.
template <class F>
__device__ Affine<F> to_affine(const Xyzz<F>& p) {
  if (is_infinity(p)) return Affine<F>{F::zero(), F::zero()};
  F inv = field_inverse(p.zz * p.zzz);
  return Affine<F>{p.x * (p.zzz * inv), p.y * (p.zz * inv)};
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
