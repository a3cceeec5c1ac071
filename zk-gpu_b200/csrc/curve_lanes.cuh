// XYZZ doubling and addition for one warp that holds a single point: the independent field
// products of each dependency level run on different lanes at once (one product's latency per
// level instead of one per product), and the results are exchanged through shared memory.
// Every lane keeps the whole (identical) state, so all branches are uniform.
//
// Products per level: doubling (dbl-2008-s-1) 2, 4, 3; addition (add-2008-s) 6, 2, 3, 3. For
// Fq2 each product is three Fq products (Karatsuba) on three lanes, so a level uses up to 18.
// The formulas and special cases are those of curve.cuh (xyzz_double, xyzz_add).
#pragma once
#include "curve.cuh"

namespace zkg {

template <class F>
struct BaseParams;
template <class P>
struct BaseParams<Fp<P>> {
  using type = P;
};

// Scratch: 32 lanes x 8 words in shared memory, owned by the warp.
struct LaneScratch {
  uint32_t* words;
};

template <class P>
__device__ __forceinline__ void lane_put(LaneScratch sm, const Fp<P>& v) {
  const unsigned lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < 8; i++) sm.words[8 * lane + i] = v.w[i];
}
template <class P>
__device__ __forceinline__ Fp<P> lane_get(LaneScratch sm, unsigned lane) {
  Fp<P> v;
#pragma unroll
  for (int i = 0; i < 8; i++) v.w[i] = sm.words[8 * lane + i];
  return v;
}

// r[k] = a[k] * b[k], k < K, lane k computing product k.
template <int K, class P>
__device__ __forceinline__ void lane_mul(const Fp<P> (&a)[K], const Fp<P> (&b)[K], Fp<P> (&r)[K], LaneScratch sm) {
  static_assert(K <= 32, "one product per lane");
  const unsigned lane = threadIdx.x & 31;
  Fp<P> x = a[0], y = b[0];
#pragma unroll
  for (int k = 1; k < K; k++) {
    if (lane == (unsigned)k) {
      x = a[k];
      y = b[k];
    }
  }
  const Fp<P> p = x * y;  // one product for the whole warp
  __syncwarp();
  lane_put(sm, p);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; k++) r[k] = lane_get<P>(sm, k);
}

// Fq2: product k takes lanes 3k (a.a * b.a), 3k+1 (a.b * b.b), 3k+2 ((a.a + a.b)(b.a + b.b)).
template <int K, class B>
__device__ __forceinline__ void lane_mul(const Fq2T<B> (&a)[K], const Fq2T<B> (&b)[K], Fq2T<B> (&r)[K],
                                         LaneScratch sm) {
  static_assert(3 * K <= 32, "three lanes per product");
  const unsigned lane = threadIdx.x & 31;
  B x = a[0].a, y = b[0].a;
#pragma unroll
  for (int k = 0; k < K; k++) {
    if (lane == (unsigned)(3 * k + 1)) {
      x = a[k].b;
      y = b[k].b;
    } else if (lane == (unsigned)(3 * k + 2)) {
      x = a[k].a + a[k].b;
      y = b[k].a + b[k].b;
    } else if (lane == (unsigned)(3 * k)) {
      x = a[k].a;
      y = b[k].a;
    }
  }
  const B p = x * y;
  __syncwarp();
  lane_put(sm, p);
  __syncwarp();
#pragma unroll
  for (int k = 0; k < K; k++) {
    const B ac = lane_get<typename BaseParams<B>::type>(sm, 3 * k);
    const B bd = lane_get<typename BaseParams<B>::type>(sm, 3 * k + 1);
    const B cross = lane_get<typename BaseParams<B>::type>(sm, 3 * k + 2);
    r[k] = Fq2T<B>{ac - bd, (cross - ac) - bd};
  }
}

// 2P (dbl-2008-s-1, a = 0), as xyzz_double.
template <class F>
__device__ __forceinline__ Xyzz<F> lane_double(const Xyzz<F>& p, LaneScratch sm) {
  const F u = dbl(p.y);
  F l1[2];
  lane_mul<2>({u, p.x}, {u, p.x}, l1, sm);  // V = U^2, X^2
  const F v = l1[0], m = dbl(l1[1]) + l1[1];
  F l2[4];
  lane_mul<4>({u, p.x, m, v}, {v, v, m, p.zz}, l2, sm);  // W, S, M^2, ZZ3
  const F w = l2[0], s = l2[1];
  const F x3 = l2[2] - dbl(s);
  F l3[3];
  lane_mul<3>({w, m, w}, {p.y, s - x3, p.zzz}, l3, sm);  // W Y, M (S - X3), ZZZ3
  return Xyzz<F>{x3, l3[1] - l3[0], l2[3], l3[2]};
}

// P + Q (add-2008-s), as xyzz_add.
template <class F>
__device__ __forceinline__ Xyzz<F> lane_add(const Xyzz<F>& p, const Xyzz<F>& q, LaneScratch sm) {
  if (is_infinity(q)) return p;
  if (is_infinity(p)) return q;
  F l1[6];
  lane_mul<6>({p.x, q.x, p.y, q.y, p.zz, p.zzz}, {q.zz, p.zz, q.zzz, p.zzz, q.zz, q.zzz}, l1, sm);
  const F u1 = l1[0], s1 = l1[2];
  const F pp = l1[1] - u1;
  const F r = l1[3] - s1;
  if (pp.is_zero()) {
    if (r.is_zero()) return lane_double(p, sm);
    return xyzz_infinity<F>();
  }
  F l2[2];
  lane_mul<2>({pp, r}, {pp, r}, l2, sm);  // PP, RR
  F l3[3];
  lane_mul<3>({pp, u1, l1[4]}, {l2[0], l2[0], l2[0]}, l3, sm);  // PPP, Q, ZZ3
  const F ppp = l3[0], qq = l3[1];
  const F x3 = (l2[1] - ppp) - dbl(qq);
  F l4[3];
  lane_mul<3>({r, s1, l1[5]}, {qq - x3, ppp, ppp}, l4, sm);  // R (Q - X3), S1 PPP, ZZZ3
  return Xyzz<F>{x3, l4[0] - l4[1], l3[2], l4[2]};
}

}  // namespace zkg
