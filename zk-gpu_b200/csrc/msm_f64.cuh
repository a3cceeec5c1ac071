// Bucket accumulation on the double-precision pipe (accumulation variants 3 and 4), G1 and G2.
//
// Same segment walk as msm_accumulate (msm_kernels.cuh) and the same mixed addition
// (madd-2008-s), but the bucket sums are kept as five 52-bit limbs per coordinate in
// Montgomery form with R = 2^260 (field_f64.cuh), whose products issue on the FP64 pipe
// (measured on B200: 65 G Fq products/s against 50 G/s for the 32-bit integer product).
// Bases stay in the library's R = 2^256 word format: a canonical word value w becomes the
// limbs of 16 w, the same element in R = 2^260 form (unreduced, below 16p). Buckets and heads
// are written back as canonical R = 2^256 words, so the merge and reduction stages are the
// integer ones. G2 runs the same formulas over Fq2 = Fq[u]/(u^2 + 1) (Karatsuba products,
// squarings from two base products), every bound below holding per component.
//
// Bounds (p < 2^254; two values whose product is below p 2^260 give a product below 2p):
//   bucket X, Y, ZZ, ZZZ < 2p;  base X2, Y2 < 16p (G1) or < 2p (G2, reduced on load);
//   U2 = X2 ZZ, S2 = Y2 ZZZ < 2p;  P = U2 - X + 2p, R = S2 - Y + 2p in (0, 4p);
//   PP, RR, PPP, Q < 2p;  D = 2Q < 4p;  X3 = RR + 6p - PPP - D in (0, 8p), reduced to [0, 2p);
//   V = Q - X3 + 2p < 4p;  Y3 = R V - Y PPP below 2p;  ZZ3 = ZZ PP, ZZZ3 = ZZZ PPP < 2p.
// P = 0 mod p (P is p, 2p or 3p) is the doubling / cancellation case; it is rare and runs the
// integer doubling on the canonical words.
#pragma once
#include <type_traits>

#include "field_f64.cuh"
#include "msm_kernels.cuh"

namespace zkg {
namespace f64 {

__device__ const MultiplesOfP g_multiples_of_p = MultiplesOfP();

// An Fq2 element (a + b u, u^2 = -1) as two limb elements.
struct Fq2D {
  FqD a, b;
};

template <class E>
struct XyzzT {
  E x, y, zz, zzz;
};

// ---- element operations, G1 (FqD) and G2 (Fq2D, componentwise unless stated)

__device__ __forceinline__ FqD e_reduce(const FqD& x, const MultiplesOfP* kp) { return fqd_reduce(x, kp); }
__device__ __forceinline__ Fq2D e_reduce(const Fq2D& x, const MultiplesOfP* kp) {
  return Fq2D{fqd_reduce(x.a, kp), fqd_reduce(x.b, kp)};
}
template <int K>
__device__ __forceinline__ FqD e_sub(const FqD& x, const FqD& y) { return fqd_sub<K>(x, y); }
template <int K>
__device__ __forceinline__ Fq2D e_sub(const Fq2D& x, const Fq2D& y) {
  return Fq2D{fqd_sub<K>(x.a, y.a), fqd_sub<K>(x.b, y.b)};
}
template <int K>
__device__ __forceinline__ FqD e_sub2(const FqD& x, const FqD& y, const FqD& z) { return fqd_sub2<K>(x, y, z); }
template <int K>
__device__ __forceinline__ Fq2D e_sub2(const Fq2D& x, const Fq2D& y, const Fq2D& z) {
  return Fq2D{fqd_sub2<K>(x.a, y.a, z.a), fqd_sub2<K>(x.b, y.b, z.b)};
}
__device__ __forceinline__ FqD e_add(const FqD& x, const FqD& y) { return fqd_add(x, y); }
__device__ __forceinline__ Fq2D e_add(const Fq2D& x, const Fq2D& y) {
  return Fq2D{fqd_add(x.a, y.a), fqd_add(x.b, y.b)};
}

// r1 = a b, r2 = c d. Fq2: Karatsuba, three pairs of base products; inputs below 4p per
// component (sums below 8p: (8p)^2 < p 2^260), outputs below 2p.
template <bool PAIRS>
__device__ __forceinline__ void e_mul2(const FqD& a, const FqD& b, const FqD& c, const FqD& d, FqD& r1, FqD& r2,
                                       const MultiplesOfP*) {
  fqd_mul2<PAIRS>(a, b, c, d, r1, r2);
}
template <bool PAIRS>
__device__ __forceinline__ void e_mul2(const Fq2D& a, const Fq2D& b, const Fq2D& c, const Fq2D& d, Fq2D& r1,
                                       Fq2D& r2, const MultiplesOfP* kp) {
  FqD ac1, ac2, bd1, bd2, cr1, cr2;
  fqd_mul2<PAIRS>(a.a, b.a, c.a, d.a, ac1, ac2);
  fqd_mul2<PAIRS>(a.b, b.b, c.b, d.b, bd1, bd2);
  fqd_mul2<PAIRS>(fqd_add(a.a, a.b), fqd_add(b.a, b.b), fqd_add(c.a, c.b), fqd_add(d.a, d.b), cr1, cr2);
  r1 = Fq2D{fqd_reduce(fqd_sub<2>(ac1, bd1), kp), fqd_reduce(fqd_sub2<4>(cr1, ac1, bd1), kp)};
  r2 = Fq2D{fqd_reduce(fqd_sub<2>(ac2, bd2), kp), fqd_reduce(fqd_sub2<4>(cr2, ac2, bd2), kp)};
}

// r1 = a^2, r2 = c^2. Fq2: (a0 + a1)(a0 - a1) and 2 a0 a1, two base products per square.
template <bool PAIRS>
__device__ __forceinline__ void e_sqr2(const FqD& a, const FqD& c, FqD& r1, FqD& r2, const MultiplesOfP*) {
  fqd_mul2<PAIRS>(a, a, c, c, r1, r2);
}
template <bool PAIRS>
__device__ __forceinline__ void e_sqr2(const Fq2D& a, const Fq2D& c, Fq2D& r1, Fq2D& r2, const MultiplesOfP* kp) {
  FqD re1, re2, ab1, ab2;
  fqd_mul2<PAIRS>(fqd_add(a.a, a.b), fqd_sub<4>(a.a, a.b), fqd_add(c.a, c.b), fqd_sub<4>(c.a, c.b), re1, re2);
  fqd_mul2<PAIRS>(a.a, a.b, c.a, c.b, ab1, ab2);
  r1 = Fq2D{re1, fqd_reduce(fqd_add(ab1, ab1), kp)};
  r2 = Fq2D{re2, fqd_reduce(fqd_add(ab2, ab2), kp)};
}

// a b - c d below 2p (a, b below 4p; c, d below 2p). G1 with one product per call: one
// reduction for both products (mont_mul_sub; 48.1 ms at 2^24 against 52.0 ms for the products
// apart); with pairs the products stay a pair (the four-operand call spills there). G2: two
// Karatsuba products, a difference and a reduction.
template <bool PAIRS>
__device__ __forceinline__ FqD e_mul_sub(const FqD& a, const FqD& b, const FqD& c, const FqD& d,
                                         const MultiplesOfP* kp) {
  if (PAIRS) {
    FqD t, u;
    fqd_mul2<true>(a, b, c, d, t, u);
    return fqd_reduce(fqd_sub<2>(t, u), kp);
  }
  return fqd_mul_sub_call(a, b, c, d);
}
template <bool PAIRS>
__device__ __forceinline__ Fq2D e_mul_sub(const Fq2D& a, const Fq2D& b, const Fq2D& c, const Fq2D& d,
                                          const MultiplesOfP* kp) {
  Fq2D t, u;
  e_mul2<PAIRS>(a, b, c, d, t, u, kp);
  return e_reduce(e_sub<2>(t, u), kp);
}

// x (below 4p per component) is 0 mod p: a one-limb filter, then the exact test.
__device__ __forceinline__ bool e_is_zero4(const FqD& x) { return fqd_maybe_zero4(x) && fqd_is_zero4(x); }
__device__ __forceinline__ bool e_is_zero4(const Fq2D& x) {
  return fqd_maybe_zero4(x.a) && fqd_maybe_zero4(x.b) && fqd_is_zero4(x.a) && fqd_is_zero4(x.b);
}

template <class E>
__device__ __forceinline__ E e_one260();
template <>
__device__ __forceinline__ FqD e_one260<FqD>() { return fqd_one260(); }
template <>
__device__ __forceinline__ Fq2D e_one260<Fq2D>() { return Fq2D{fqd_one260(), FqD{{0.0, 0.0, 0.0, 0.0, 0.0}}}; }

// ---- conversions to and from the library's word format (R = 2^256, canonical)

template <class E>
struct Words;  // integer element type with the same word layout
template <>
struct Words<FqD> {
  using type = FqC;
};
template <>
struct Words<Fq2D> {
  using type = Fq2C;
};

__device__ __forceinline__ FqD fqd_from(const FqC& a) {
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w[i] = a.w[i];
  return fqd_from_words_x16(w);  // below 16p
}
// A base coordinate, ready for the products: G1 feeds the value below 16p straight in (a
// product of it with a value below 2p stays under p 2^260); G2 reduces it below 2p first,
// since the Karatsuba sums add two coordinates.
__device__ __forceinline__ FqD e_base(const FqC& a, const MultiplesOfP*) { return fqd_from(a); }
__device__ __forceinline__ Fq2D e_base(const Fq2C& a, const MultiplesOfP* kp) {
  return Fq2D{fqd_reduce(fqd_from(a.a), kp), fqd_reduce(fqd_from(a.b), kp)};
}
__device__ __forceinline__ FqD e_from(const FqC& a, const MultiplesOfP* kp) { return fqd_reduce(fqd_from(a), kp); }
__device__ __forceinline__ Fq2D e_from(const Fq2C& a, const MultiplesOfP* kp) {
  return Fq2D{fqd_reduce(fqd_from(a.a), kp), fqd_reduce(fqd_from(a.b), kp)};
}

struct Words8 {
  uint32_t w[8];
};

// Canonical R = 2^256 words of an R = 2^260 element below 2p (out of line: cold paths only).
static __device__ __noinline__ Words8 fqd_words_call(FqD a) {
  Words8 r;
  fqd_to_words(a, r.w);
  return r;
}

__device__ __forceinline__ FqC e_words(const FqD& a) {
  const Words8 v = fqd_words_call(a);
  FqC r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = v.w[i];
  return r;
}
__device__ __forceinline__ Fq2C e_words(const Fq2D& a) { return Fq2C{e_words(a.a), e_words(a.b)}; }

// Canonical R = 2^256 words (x, y, zz, zzz), or all zeros for infinity.
template <class E>
__device__ __forceinline__ void store_xyzzd(uint32_t* p, const XyzzT<E>& a, bool empty) {
  using W = typename Words<E>::type;
  if (empty) {
    store_xyzz(p, xyzz_infinity<W>());
  } else {
    store_xyzz(p, Xyzz<W>{e_words(a.x), e_words(a.y), e_words(a.zz), e_words(a.zzz)});
  }
}

// 2 acc through the integer doubling (rare: equal points in one bucket). The accumulator never
// has its address taken, so it stays in registers. Returns false for infinity.
template <class E>
__device__ __forceinline__ bool xyzzd_double_slow(XyzzT<E>& acc, const MultiplesOfP* kp) {
  using W = typename Words<E>::type;
  const Xyzz<W> d = xyzz_double_call(Xyzz<W>{e_words(acc.x), e_words(acc.y), e_words(acc.zz), e_words(acc.zzz)});
  if (d.zz.is_zero()) return false;
  acc = XyzzT<E>{e_from(d.x, kp), e_from(d.y, kp), e_from(d.zz, kp), e_from(d.zzz, kp)};
  return true;
}

// Where a thread's bucket accumulator lives. AccRegs: registers (G1). AccSmem: the block's
// shared memory, limb-major over its 128 threads (slot k of thread t at base[k * 128 + t]), each
// coordinate read right before it is used, so the addition's registers hold only its
// temporaries (a G2 accumulator is 40 doubles, which in registers push the kernel into spills).
template <class E>
struct AccRegs {
  XyzzT<E> v;
  __device__ __forceinline__ E x() const { return v.x; }
  __device__ __forceinline__ E y() const { return v.y; }
  __device__ __forceinline__ E zz() const { return v.zz; }
  __device__ __forceinline__ E zzz() const { return v.zzz; }
  __device__ __forceinline__ XyzzT<E> get() const { return v; }
  __device__ __forceinline__ void set(const XyzzT<E>& a) { v = a; }
};
__device__ __forceinline__ void slots_ld(const double* p, FqD& e) {
#pragma unroll
  for (int k = 0; k < 5; k++) e.l[k] = p[k * 128];
}
__device__ __forceinline__ void slots_ld(const double* p, Fq2D& e) {
  slots_ld(p, e.a);
  slots_ld(p + 5 * 128, e.b);
}
__device__ __forceinline__ void slots_st(double* p, const FqD& e) {
#pragma unroll
  for (int k = 0; k < 5; k++) p[k * 128] = e.l[k];
}
__device__ __forceinline__ void slots_st(double* p, const Fq2D& e) {
  slots_st(p, e.a);
  slots_st(p + 5 * 128, e.b);
}
template <class E>
struct AccSmem {
  static constexpr int N = sizeof(E) / sizeof(double);  // doubles per element
  double* base;  // &slots[threadIdx.x]
  __device__ __forceinline__ E ld(int coord) const {
    E e;
    slots_ld(base + coord * N * 128, e);
    return e;
  }
  __device__ __forceinline__ void st(int coord, const E& e) { slots_st(base + coord * N * 128, e); }
  __device__ __forceinline__ E x() const { return ld(0); }
  __device__ __forceinline__ E y() const { return ld(1); }
  __device__ __forceinline__ E zz() const { return ld(2); }
  __device__ __forceinline__ E zzz() const { return ld(3); }
  __device__ __forceinline__ XyzzT<E> get() const { return XyzzT<E>{ld(0), ld(1), ld(2), ld(3)}; }
  __device__ __forceinline__ void set(const XyzzT<E>& a) {
    st(0, a.x);
    st(1, a.y);
    st(2, a.zz);
    st(3, a.zzz);
  }
};

// acc += (bx, by) with acc not at infinity (madd-2008-s), with the bounds stated at the top of
// this file. Returns false when the sum is infinity.
template <class E, bool PAIRS, class Acc>
__device__ __forceinline__ bool xyzzd_add_affine(Acc& acc, const E& bx, const E& by, const MultiplesOfP* kp) {
  E u2, s2;
  e_mul2<PAIRS>(bx, acc.zz(), by, acc.zzz(), u2, s2, kp);
  const E pp = e_sub<2>(u2, acc.x());
  const E r = e_sub<2>(s2, acc.y());
  if (e_is_zero4(pp)) {
    if (!e_is_zero4(r)) return false;
    XyzzT<E> t = acc.get();
    const bool live = xyzzd_double_slow(t, kp);
    if (live) acc.set(t);
    return live;
  }
  E ppsq, rr, ppp, q;
  e_sqr2<PAIRS>(pp, r, ppsq, rr, kp);
  e_mul2<PAIRS>(pp, ppsq, acc.x(), ppsq, ppp, q, kp);
  const E d = e_add(q, q);
  const E x3 = e_reduce(e_sub2<6>(rr, ppp, d), kp);
  const E v = e_sub<2>(q, x3);
  const E y3 = e_mul_sub<PAIRS>(r, v, acc.y(), ppp, kp);  // R V - Y PPP
  E zz3, zzz3;
  e_mul2<PAIRS>(acc.zz(), ppsq, acc.zzz(), ppp, zz3, zzz3, kp);
  acc.set(XyzzT<E>{x3, y3, zz3, zzz3});
  return true;
}

}  // namespace f64

// msm_accumulate (msm_kernels.cuh) with the bucket arithmetic in double-precision limbs: E =
// FqD (G1) or Fq2D (G2); PAIRS: two products per out-of-line call, else one. The next base is
// fetched into shared memory with cp.async (two slots per thread) while the current addition
// runs, so the prefetch holds no registers (G1: 50.9 ms at 2^24 against 52.9 ms fetching into
// registers). Three blocks of 128 threads per SM (168 registers) measured faster than four (128
// registers and ~100 bytes of spills per thread: 48.5 against 48.0 ms at 2^24). G2 keeps the
// accumulators in shared memory (AccSmem; in registers they are 80 of them and the kernel
// spilled): 55.9 / 63.0 ms at 2^22 for one / two products per call, from 67 / 73, still behind
// the integer pairs (47.3 ms); at three blocks per SM it spills again.
// G1 with SMEM_ACC (accumulation variants 5 and 6): the accumulator in shared memory as for G2,
// which frees its 40 registers for a fourth block per SM (128 registers).
template <class E, bool PAIRS, bool SMEM_ACC = !std::is_same<E, f64::FqD>::value>
__global__ void __launch_bounds__(128, std::is_same<E, f64::FqD>::value ? (SMEM_ACC ? 4 : 3) : 2)
    msm_accumulate_f64(const uint32_t* __restrict__ bases, const uint32_t* __restrict__ bases2, uint32_t split,
                       const uint32_t* __restrict__ sorted,
                       const uint32_t* __restrict__ slot_start, uint32_t num_slots, uint32_t seg_len,
                       uint32_t* __restrict__ buckets, uint32_t* __restrict__ heads,
                       uint32_t* __restrict__ head_keys) {
  using namespace f64;
  using W = typename Words<E>::type;
  constexpr int XW = PointWords<W>::xyzz;
  constexpr int AW = PointWords<W>::affine;
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

  using Acc = typename std::conditional<SMEM_ACC, AccSmem<E>, AccRegs<E>>::type;
  extern __shared__ __align__(16) double acc_slots[];  // SMEM_ACC: 4 * AccSmem<E>::N * 128 doubles
  Acc acc;
  if constexpr (SMEM_ACC) acc.base = acc_slots + threadIdx.x;
  bool empty = true;
  __shared__ __align__(16) uint32_t stage[2][128][AW];
  auto stage_base = [&](uint32_t slot, uint32_t e) {  // x then y; points from split on in bases2
    const uint32_t pt = e & ~kNegBit;
    const uint4* g = reinterpret_cast<const uint4*>(pt < split ? bases + (size_t)pt * AW
                                                               : bases2 + (size_t)(pt - split) * AW);
    const uint32_t sa = (uint32_t)__cvta_generic_to_shared(&stage[slot][threadIdx.x][0]);
#pragma unroll
    for (int k = 0; k < AW / 4; k++)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa + 16 * k), "l"(g + k) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  uint32_t entry = __ldg(&sorted[p0]);
  uint32_t cur_entry = entry, slot = 0;
  stage_base(0, entry);
  for (uint32_t p = p0; p < p1; p++) {
    if (p + 1 < p1) {
      entry = __ldg(&sorted[p + 1]);
      stage_base(slot ^ 1, entry);
      asm volatile("cp.async.wait_group 1;" ::: "memory");  // this point's copy has landed
    } else {
      asm volatile("cp.async.wait_group 0;" ::: "memory");
    }
    Affine<W> cur = load_affine<W>(&stage[slot][threadIdx.x][0]);
    if (cur_entry & kNegBit) cur.y = neg(cur.y);
    cur_entry = entry;
    slot ^= 1;
    if (p == end) {
      if (head) {
        store_xyzzd(heads + (size_t)t * XW, acc.get(), empty);
        head_key = s;
        head = false;
      } else {
        store_xyzzd(buckets + (size_t)s * XW, acc.get(), empty);
      }
      empty = true;
      uint32_t s2 = s + 1;
      if (__ldg(&slot_start[s2 + 1]) <= p) s2 = last_leq(slot_start, s2, num_slots, p);
      s = s2;
      end = __ldg(&slot_start[s + 1]);
    }
    if (is_infinity(cur)) continue;
    const E bx = e_base(cur.x, kp), by = e_base(cur.y, kp);
    if (empty) {
      acc.set(XyzzT<E>{e_reduce(bx, kp), e_reduce(by, kp), e_one260<E>(), e_one260<E>()});
      empty = false;
    } else {
      empty = !xyzzd_add_affine<E, PAIRS>(acc, bx, by, kp);
    }
  }
  if (head) {
    store_xyzzd(heads + (size_t)t * XW, acc.get(), empty);
    head_key = s;
  } else {
    store_xyzzd(buckets + (size_t)s * XW, acc.get(), empty);
  }
  head_keys[t] = head_key;
}

}  // namespace zkg
