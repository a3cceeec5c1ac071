// MSM device kernels (signed-digit Pippenger), templated on the coordinate field
// (Fq for G1, Fq2 for G2).
//
// Pipeline for one run (reference stage in brackets):
//   1. recode + count   per point, W signed c-bit digits; warp-aggregated histogram of
//                       (window, |digit|) slots                    [msm_digits.wgsl, count]
//   2. scan             exclusive prefix sum over all W*B slots -> slot_start, cursor
//                                                                  [msm_scan.wgsl]
//   3. recode + scatter point index (sign in bit 31) written to its slot's range, one u32 per
//                       nonzero digit, warp-aggregated cursors     [msm_digits.wgsl, scatter]
//   4. accumulate       the sorted array is cut into equal segments of L entries, one per
//                       thread, regardless of bucket boundaries: every thread does exactly L
//                       mixed additions, so skewed bucket sizes cannot unbalance the warps.
//                       A bucket that starts in a segment is written by that segment's thread;
//                       the parts of a bucket that continue into later segments ("heads")
//                       are emitted per segment with the bucket's slot as key.
//                                                                  [msm_accumulate.wgsl]
//   5. merge levels     heads with equal keys are contiguous; each level sums runs of up to
//                       L1 of them, adds runs that start in its range into the bucket, and
//                       passes runs that continue from the previous range to the next level
//                       (log_L1 levels)                            [msm_merge/finalize.wgsl]
//   6. reduce levels    per window S_w = sum_b (b+1) * bucket_b, by chunked running sums:
//                       chunk k of 16 buckets gives tot_k = sum_j (j+1) B_j and run_k =
//                       sum_j B_j; S_w = sum_k tot_k + 16 * sum_k k * run_k, and the second
//                       sum is the same problem over run_1.. (next level)
//                                                                  [msm_reduce_chunks.wgsl,
//                                                                   msm_sum.wgsl]
//   7. window sums      per window, sum each level's tot_k and fold levels (x16 between)
//   8. combine          Horner over windows, c doublings each      [msm_combine.wgsl]
#pragma once
#include "curve.cuh"
#include "curve_lanes.cuh"
#include "msm_common.hpp"

namespace zkg {


template <class F>
struct PointWords {
  static constexpr int affine = 2 * FieldWords<F>::value;
  static constexpr int xyzz = 4 * FieldWords<F>::value;
};

// ------------------------------------------------------------------ recoding

// Window w's raw c bits of the scalar (8 LE words). c <= 20 < 32, so two words suffice.
__device__ __forceinline__ uint32_t window_bits(const uint32_t s[8], uint32_t pos, uint32_t c) {
  uint32_t word = pos >> 5, off = pos & 31;
  uint32_t v = 0;
  if (word < 8) v = s[word] >> off;
  if (off + c > 32 && word + 1 < 8) v |= s[word + 1] << (32 - off);
  return v & ((1u << c) - 1);
}

__device__ __forceinline__ void load_scalar(const uint32_t* scalars, size_t i, uint32_t s[8]) {
  const uint4* p = reinterpret_cast<const uint4*>(scalars + 8 * i);
  uint4 lo = __ldg(p), hi = __ldg(p + 1);
  s[0] = lo.x; s[1] = lo.y; s[2] = lo.z; s[3] = lo.w;
  s[4] = hi.x; s[5] = hi.y; s[6] = hi.z; s[7] = hi.w;
}

// Digit recoding of msm_digits.wgsl:19-37: v = window + carry; v >= 2^(c-1) gives the
// negative digit v - 2^c (magnitude 2^c - v) and a carry into the next window. Returns the
// slot (w * B + |digit| - 1) or kNoKey for a zero digit; *neg gets the sign.
struct Recoder {
  uint32_t s[8];
  uint32_t carry = 0;
  __device__ __forceinline__ uint32_t next(uint32_t w, uint32_t c, uint32_t half, bool* neg) {
    uint32_t v = window_bits(s, w * c, c) + carry;
    carry = 0;
    uint32_t mag = v;
    *neg = false;
    if (v >= half) {
      mag = (1u << c) - v;
      *neg = true;
      carry = 1;
    }
    return mag ? w * half + mag - 1 : kNoKey;
  }
};

// Recoding of a GLV half (127-bit magnitude in four words; the words are picked by selects, so
// two of these stay in registers in one thread).
struct GlvRecoder {
  uint32_t s[4];
  uint32_t carry = 0;
  __device__ __forceinline__ uint32_t word(uint32_t i) const {
    return i == 0 ? s[0] : i == 1 ? s[1] : i == 2 ? s[2] : i == 3 ? s[3] : 0u;
  }
  __device__ __forceinline__ uint32_t window_bits(uint32_t pos, uint32_t width) const {
    const uint32_t wd = pos >> 5, off = pos & 31;
    uint32_t v = word(wd) >> off;
    if (off + width > 32) v |= word(wd + 1) << (32 - off);
    return v & ((1u << width) - 1);
  }
  // Recoder::next for a window of `width` bits starting at bit `pos` (width <= c: the GLV
  // windows), the digit negated when `flip` (a negative half-scalar: its digits are those of |k| with the
  // sign turned). A flipped half is recoded with v > 2^(width-1) negative instead of >=, so its
  // digits lie in (-2^(width-1), 2^(width-1)] and, turned, in [-2^(width-1), 2^(width-1)) like
  // every other digit: the positive magnitude 2^(c-1), whose 16-bit code is kRankZero at c = 16,
  // never occurs.
  __device__ __forceinline__ uint32_t next_at(uint32_t w, uint32_t pos, uint32_t width, uint32_t half, bool flip,
                                              bool* neg) {
    const uint32_t v = window_bits(pos, width) + carry;
    const uint32_t h = 1u << (width - 1);
    carry = 0;
    uint32_t mag = v;
    bool neg_d = false;
    if (flip ? v > h : v >= h) {
      mag = (1u << width) - v;
      neg_d = true;
      carry = 1;
    }
    *neg = neg_d != flip;
    return mag ? w * half + mag - 1 : kNoKey;
  }
};

// GLV windows: the 128 bits of the halves split as evenly as possible over W windows, the first
// 128 mod W of them floor(128 / W) + 1 bits wide and the rest floor(128 / W) (at most c bits
// each, since W = ceil(128 / c)). Equal c-bit windows would leave the top one with as little as
// 0.2 significant bits (|k| < 2^126.2), whose few buckets would take every entry's counting
// atomic; here every window keeps at least floor(128 / W) - 1.8 bits, and the top one still
// cannot carry out.
__device__ __forceinline__ uint32_t glv_window_pos(uint32_t w, uint32_t windows) {
  const uint32_t base = 128u / windows, extra = 128u % windows;
  return w * base + (w < extra ? w : extra);
}
__device__ __forceinline__ uint32_t glv_window_width(uint32_t w, uint32_t windows) {
  return 128u / windows + (w < 128u % windows ? 1u : 0u);
}

// Lanes of a warp that share a slot, for one atomic per group. AGG 0: every group
// (__match_any_sync); 1: only the group of the first lane that has a slot (one shuffle and one
// ballot: skewed inputs put most repeats into one hot slot per window); 2: none; 3: the group of
// the first lane whose right neighbour has the same slot (a slot held by a sizeable share of
// the warp almost always shows up in an adjacent pair; uniform digits almost never do, and
// then no group forms). Lanes without a slot (kNoKey) get an empty mask.
template <int AGG>
__device__ __forceinline__ unsigned slot_peers(uint32_t slot) {
  const unsigned lane = threadIdx.x & 31;
  const unsigned active = __activemask();
  if (AGG == 0) {
    const unsigned m = __match_any_sync(active, slot);  // every lane of the mask takes part
    return slot == kNoKey ? 0u : m;
  }
  if (AGG == 1) {
    const unsigned valid = __ballot_sync(active, slot != kNoKey);
    if (!valid) return 0u;
    const int first = __ffs(valid) - 1;
    const uint32_t hot = __shfl_sync(active, slot, first);
    const unsigned group = __ballot_sync(active, slot == hot) & valid;
    if (slot == kNoKey) return 0u;
    return slot == hot ? group : (1u << lane);
  }
  if (AGG == 3) {
    const unsigned valid = __ballot_sync(active, slot != kNoKey);
    const uint32_t right = __shfl_down_sync(active, slot, 1);
    const unsigned pairs = __ballot_sync(active, slot != kNoKey && lane < 31 && slot == right);
    if (slot == kNoKey) return 0u;
    if (!pairs) return 1u << lane;
    const uint32_t hot = __shfl_sync(valid | pairs, slot, __ffs(pairs) - 1);
    const unsigned group = __ballot_sync(valid, slot == hot);
    return slot == hot ? group : (1u << lane);
  }
  return slot == kNoKey ? 0u : (1u << lane);
}

// Pass 1: histogram of (window, bucket) slots; lanes of a warp that hit the same slot are
// merged into one atomic as slot_peers<AGG> groups them (equal scalars, zero-heavy or
// r-1-heavy inputs hammer single slots).
template <int AGG>
__global__ void msm_count(const uint32_t* __restrict__ scalars, size_t n, uint32_t c, uint32_t windows,
                          uint32_t* __restrict__ counts) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool live = i < n;
  Recoder rc;
  if (live) load_scalar(scalars, i, rc.s);
  uint32_t half = 1u << (c - 1);
  const unsigned lane = threadIdx.x & 31;
  for (uint32_t w = 0; w < windows; w++) {
    bool neg;
    uint32_t slot = live ? rc.next(w, c, half, &neg) : kNoKey;
    const unsigned peers = slot_peers<AGG>(slot);
    if (peers && (int)lane == __ffs(peers) - 1) atomicAdd(&counts[slot], (uint32_t)__popc(peers));
  }
}

// Pass 3: scatter point indices (sign in bit 31) into slot order. Within a slot the order is
// whatever the atomics give; bucket sums are exact, so the result does not depend on it.
// Issuing 4 or 8 windows' atomics together measured 1-3% slower at 2^24, so the pass is not
// bound by the atomics' round trips; its scattered 4-byte stores (a 32-byte sector each) are
// the likely bound.
template <int AGG>
__global__ void msm_scatter(const uint32_t* __restrict__ scalars, size_t n, uint32_t c, uint32_t windows,
                            uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool live = i < n;
  Recoder rc;
  if (live) load_scalar(scalars, i, rc.s);
  uint32_t half = 1u << (c - 1);
  const unsigned lane = threadIdx.x & 31;
  for (uint32_t w = 0; w < windows; w++) {
    bool neg = false;
    uint32_t slot = live ? rc.next(w, c, half, &neg) : kNoKey;
    const unsigned peers = slot_peers<AGG>(slot);
    if (AGG == 2) {
      if (peers) sorted[atomicAdd(&cursor[slot], 1u)] = (uint32_t)i | (neg ? kNegBit : 0u);
      continue;
    }
    // every lane takes part in the shuffle below: groups are disjoint, each with its own leader
    const int leader = peers ? __ffs(peers) - 1 : (int)lane;
    uint32_t base = 0;
    if (peers && (int)lane == leader) base = atomicAdd(&cursor[slot], (uint32_t)__popc(peers));
    base = __shfl_sync(__activemask(), base, leader);
    if (peers) sorted[base + __popc(peers & ((1u << lane) - 1))] = (uint32_t)i | (neg ? kNegBit : 0u);
  }
}

// ------------------------------------------------------------------ GLV split (G1)
//
// BN254 G1 has the endomorphism phi(x, y) = (beta x, y), beta a cube root of unity in Fq, and
// phi(P) = lambda P for every P of G1 (a group of prime order r) with lambda the matching cube
// root of unity in Fr. A scalar splits as k = k1 + k2 lambda (mod r) with short k1, k2
// (Gallant, Lambert, Vanstone, CRYPTO 2001), so sum k_i P_i = sum (k1_i P_i + k2_i phi(P_i)): an
// MSM over 2n points whose scalars have 127-bit magnitudes, half the windows of the 254-bit one.
//
// Lattice split: v1 = (a1, b1), v2 = (a2, b2) are short vectors with a + b lambda = 0 (mod r) and
// a1 b2 - a2 b1 = r (the extended Euclidean algorithm on (r, lambda)); c1 = round(b2 k / r), c2 =
// round(-b1 k / r), k1 = k - c1 a1 - c2 a2, k2 = -c1 b1 - c2 b2. The roundings use g1 =
// round(2^256 b2 / r) and g2 = round(2^256 (-b1) / r): c = floor((k g + 2^255) / 2^256) is within
// 1/2 + k / 2^257 < 5/8 of the exact quotient for k < r, so (k1, k2) = -e1 v1 - e2 v2 with |e1|,
// |e2| < 5/8, and |k1|, |k2| < 5/8 (a1 + a2) < 2^126.2 (a2 = -b1 < 2^64, b2 < 2^127). Signed
// c-bit digits of such a magnitude need ceil(128 / c) windows: the top window's bits stay below
// 2^(c - 1.8), so its digit never carries out.
namespace glv {
__device__ constexpr uint64_t kR[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                            0x30644e72e131a029ull};
__device__ constexpr uint64_t kA1[2] = {0x8211bbeb7d4f1128ull, 0x6f4d8248eeb859fcull};
__device__ constexpr uint64_t kB2[2] = {0x0be4e1541221250bull, 0x6f4d8248eeb859fdull};
__device__ constexpr uint64_t kShort[1] = {0x89d3256894d213e3ull};  // a2 = -b1
__device__ constexpr uint64_t kG1[3] = {0x5398fd0300ff6565ull, 0x4ccef014a773d2d2ull, 0x2ull};
__device__ constexpr uint64_t kG2[2] = {0xd91d232ec7e0b3d7ull, 0x2ull};
// beta = 0x30644e72e131a0295e6dd9e7e0acccb0c28f069fbb966e3de4bd44e5607cfd48 (beta^3 = 1 mod q,
// paired with lambda = 0x30644e72e131a029048b6e193fd84104cc37a73fec2bc5e9b8ca0b2d36636f23 mod
// r), here times 2^256 mod q (Montgomery form).
__device__ constexpr uint32_t kBetaMont[8] = {0x13e80b9cu, 0x3350c88eu, 0xdb5e56b9u, 0x7dce557cu,
                                   0xb615564au, 0x6001b4b8u, 0x020217e0u, 0x2682e617u};

// The low L limbs of a * b (64-bit limbs, little-endian).
template <int L, int LA, int LB>
__device__ __forceinline__ void mul_lo(const uint64_t (&a)[LA], const uint64_t (&b)[LB], uint64_t (&r)[L]) {
#pragma unroll
  for (int k = 0; k < L; k++) r[k] = 0;
#pragma unroll
  for (int i = 0; i < LA; i++) {
    uint64_t carry = 0;
#pragma unroll
    for (int j = 0; j < LB; j++) {
      if (i + j < L) {
        const uint64_t lo = a[i] * b[j], hi = __umul64hi(a[i], b[j]);
        uint64_t t = r[i + j] + lo;
        uint64_t cy = t < lo;
        t += carry;
        cy += t < carry;
        r[i + j] = t;
        carry = hi + cy;  // r + a b + carry < 2^128: no overflow
      }
    }
    if (i + LB < L) r[i + LB] = carry;
  }
}

// a - b mod 2^(64 L).
template <int L>
__device__ __forceinline__ void sub_mod(uint64_t (&a)[L], const uint64_t (&b)[L]) {
  uint64_t borrow = 0;
#pragma unroll
  for (int i = 0; i < L; i++) {
    const uint64_t x = a[i] - b[i];
    const uint64_t b1 = a[i] < b[i];
    a[i] = x - borrow;
    borrow = b1 | (x < borrow);
  }
}

// floor((k g + 2^255) / 2^256), taking the LC limbs of the quotient.
template <int LG, int LC>
__device__ __forceinline__ void round_quotient(const uint64_t (&k)[4], const uint64_t (&g)[LG], uint64_t (&c)[LC]) {
  uint64_t p[4 + LG];
  mul_lo<4 + LG>(k, g, p);
  const uint64_t t = p[3] + (1ull << 63);
  uint64_t carry = t < p[3];
#pragma unroll
  for (int i = 4; i < 4 + LG; i++) {
    p[i] += carry;
    carry = carry && p[i] == 0;
  }
#pragma unroll
  for (int i = 0; i < LC; i++) c[i] = p[4 + i];
}

// |v| (a signed 192-bit value, |v| < 2^127) into out (words 0..3; 4..7 zero); whether v < 0.
__device__ __forceinline__ bool store_half(uint64_t (&v)[3], uint32_t out[8]) {
  const bool neg = v[2] >> 63;
  if (neg) {
    uint64_t m[3] = {0, 0, 0};
    sub_mod(m, v);
    v[0] = m[0];
    v[1] = m[1];
  }
  out[0] = (uint32_t)v[0];
  out[1] = (uint32_t)(v[0] >> 32);
  out[2] = (uint32_t)v[1];
  out[3] = (uint32_t)(v[1] >> 32);
#pragma unroll
  for (int i = 4; i < 8; i++) out[i] = 0;
  return neg;
}

// s (8 words, any 256-bit value; reduced mod r first, which changes no multiple of a point of
// G1) -> |k1| in k1, |k2| in k2 (words 0..3, words 4..7 zero) and their signs.
__device__ __forceinline__ void split(const uint32_t s[8], uint32_t k1[8], bool& neg1, uint32_t k2[8], bool& neg2) {
  uint64_t k[4];
#pragma unroll
  for (int i = 0; i < 4; i++) k[i] = s[2 * i] | (uint64_t)s[2 * i + 1] << 32;
#pragma unroll
  for (int t = 0; t < 5; t++) {  // 2^256 < 6 r
    uint64_t d[4] = {k[0], k[1], k[2], k[3]};
    uint64_t borrow = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint64_t x = d[i] - kR[i];
      const uint64_t b1 = d[i] < kR[i];
      d[i] = x - borrow;
      borrow = b1 | (x < borrow);
    }
    if (!borrow) {
#pragma unroll
      for (int i = 0; i < 4; i++) k[i] = d[i];
    }
  }
  uint64_t c1[2], c2[1];
  round_quotient(k, kG1, c1);  // < b2 + 1 < 2^127
  round_quotient(k, kG2, c2);  // < -b1 + 1 < 2^64
  uint64_t v[3] = {k[0], k[1], k[2]}, t[3];  // k1 = k - c1 a1 - c2 a2
  mul_lo<3>(c1, kA1, t);
  sub_mod(v, t);
  mul_lo<3>(c2, kShort, t);
  sub_mod(v, t);
  neg1 = store_half(v, k1);
  mul_lo<3>(c1, kShort, v);  // k2 = c1 (-b1) - c2 b2
  mul_lo<3>(c2, kB2, t);
  sub_mod(v, t);
  neg2 = store_half(v, k2);
}

// One half of split: s -> |k1| (second = false) or |k2| (second = true), returning its sign.
__device__ __forceinline__ bool split_half(uint32_t s[8], bool second) {
  uint32_t h1[8], h2[8];
  bool n1, n2;
  split(s, h1, n1, h2, n2);
#pragma unroll
  for (int i = 0; i < 8; i++) s[i] = second ? h2[i] : h1[i];
  return second ? n2 : n1;
}
}  // namespace glv

// phi(P_i) = (beta x_i, y_i) for the n bases (affine, Montgomery form; infinity, (0, 0), stays
// (0, 0)): the bases of GLV entries n..2n-1. Entries 0..n-1 read P_i from the caller's bases, and
// every entry's half-scalar sign is in its digits.
__global__ void msm_glv_phi(const uint32_t* __restrict__ bases, size_t n, uint32_t* __restrict__ phi) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Fq beta;
#pragma unroll
  for (int k = 0; k < 8; k++) beta.w[k] = glv::kBetaMont[k];
  const uint4* src = reinterpret_cast<const uint4*>(bases + 16 * i);
  store_fe(phi + 16 * i, load_fe<Fq>(bases + 16 * i) * beta);
  uint4* dst = reinterpret_cast<uint4*>(phi + 16 * i);
  dst[2] = __ldg(src + 2);
  dst[3] = __ldg(src + 3);
}

// ------------------------------------------------------------------ ranked counting sort
//
// The same sort in two passes without scattered stores over the whole sorted array:
//   msm_rank  recodes each scalar once; the warp-aggregated atomic that counts a digit also
//             returns its rank within its slot; the digit (bucket | sign << 15, kRankZero for a
//             zero digit; 16 bits) and the rank (32 bits) go to window-major arrays (entry
//             w * n + i) with coalesced streaming stores.
//   msm_place after the scan, walks the entries window by window: sorted[slot_start + rank] =
//             point index | sign. A window's slots span ~4n bytes of the sorted array, so the
//             4-byte stores of the blocks in flight meet in L2 (the scalar-major scatter touches
//             all windows' ranges at once: 1 GiB at 2^24), and no pass needs a second atomic.
// For c <= 16 (15-bit buckets).
constexpr uint32_t kRankZero = 0x7fffu;  // a positive bucket 2^15 - 1 never occurs for c <= 16

// fixed (fixed-base tables: one set of buckets for all windows, see msm_place): the digit of
// window w counts in bucket slot |d| - 1 instead of w * 2^(c-1) + |d| - 1.
template <int AGG>
__global__ void msm_rank(const uint32_t* __restrict__ scalars, size_t n, uint32_t c, uint32_t windows, int fixed,
                         uint32_t* __restrict__ counts, uint16_t* __restrict__ digits,
                         uint32_t* __restrict__ ranks) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < n;
  Recoder rc;
  if (live) load_scalar(scalars, i, rc.s);
  const uint32_t half = 1u << (c - 1);
  const unsigned lane = threadIdx.x & 31;
  // Windows four at a time: the four counting atomics (each returns the entry's rank) are in
  // flight together before any result is used.
  constexpr int kBatch = 4;
  for (uint32_t w0 = 0; w0 < windows; w0 += kBatch) {
    uint32_t slot[kBatch], base[kBatch];
    unsigned peers[kBatch];
    bool neg[kBatch];
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const uint32_t w = w0 + k;
      slot[k] = kNoKey;
      neg[k] = false;
      if (w < windows) {  // uniform across the warp
        if (live) slot[k] = rc.next(w, c, half, &neg[k]);
        if (fixed && slot[k] != kNoKey) slot[k] -= w * half;
        peers[k] = slot_peers<AGG>(slot[k]);
        base[k] = 0;
        if (peers[k] && (int)lane == __ffs(peers[k]) - 1) base[k] = atomicAdd(&counts[slot[k]], (uint32_t)__popc(peers[k]));
      }
    }
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const uint32_t w = w0 + k;
      if (w >= windows) break;
      const int leader = peers[k] ? __ffs(peers[k]) - 1 : (int)lane;
      const uint32_t b = __shfl_sync(0xffffffffu, base[k], leader);
      if (!live) continue;
      uint32_t code = kRankZero;
      const size_t e = (size_t)w * n + i;
      if (peers[k]) {
        code = (fixed ? slot[k] : slot[k] - w * half) | (neg[k] ? 0x8000u : 0u);
        __stcs(ranks + e, b + __popc(peers[k] & ((1u << lane) - 1)));  // streamed: read once by msm_place
      }
      __stcs(digits + e, (unsigned short)code);
    }
  }
}

// The GLV counting pass, one thread per scalar: thread i splits scalar i once (glv::split) and
// recodes both halves, point i (|k1|, base P_i) and point scalar_n + i (|k2|, base phi(P_i)),
// each half's sign folded into its digits. Entries are window-major with the two halves of a
// scalar side by side (column 2i + h): the placing pass then walks them in the order this pass
// ranked them (columns in point order put each slot's ranks of one half after the other half's
// and cost 0.6 ms more placement at 2^24). Two windows per batch: four counting atomics in
// flight.
template <int AGG>
__global__ void msm_rank_glv(const uint32_t* __restrict__ scalars, size_t scalar_n, uint32_t c, uint32_t windows,
                             uint32_t* __restrict__ counts, uint16_t* __restrict__ digits,
                             uint32_t* __restrict__ ranks) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = i < scalar_n;
  const size_t n = 2 * scalar_n;
  GlvRecoder rc[2];
  bool flip[2] = {false, false};
  if (live) {
    uint32_t s[8], h1[8], h2[8];
    load_scalar(scalars, i, s);
    glv::split(s, h1, flip[0], h2, flip[1]);
#pragma unroll
    for (int j = 0; j < 4; j++) {
      rc[0].s[j] = h1[j];
      rc[1].s[j] = h2[j];
    }
  }
  const uint32_t half = 1u << (c - 1);
  const unsigned lane = threadIdx.x & 31;
  constexpr int kBatch = 2;
  for (uint32_t w0 = 0; w0 < windows; w0 += kBatch) {
    uint32_t slot[kBatch][2], base[kBatch][2];
    unsigned peers[kBatch][2];
    bool neg[kBatch][2];
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const uint32_t w = w0 + k;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        slot[k][h] = kNoKey;
        neg[k][h] = false;
        peers[k][h] = 0;
        base[k][h] = 0;
        if (w < windows) {  // uniform across the warp
          if (live)
            slot[k][h] = rc[h].next_at(w, glv_window_pos(w, windows), glv_window_width(w, windows), half, flip[h],
                                       &neg[k][h]);
          peers[k][h] = slot_peers<AGG>(slot[k][h]);
          if (peers[k][h] && (int)lane == __ffs(peers[k][h]) - 1)
            base[k][h] = atomicAdd(&counts[slot[k][h]], (uint32_t)__popc(peers[k][h]));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kBatch; k++) {
      const uint32_t w = w0 + k;
      if (w < windows) {
        uint32_t code[2], rank[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int leader = peers[k][h] ? __ffs(peers[k][h]) - 1 : (int)lane;
          const uint32_t b = __shfl_sync(0xffffffffu, base[k][h], leader);
          code[h] = peers[k][h] ? (slot[k][h] - w * half) | (neg[k][h] ? 0x8000u : 0u) : kRankZero;
          rank[h] = b + __popc(peers[k][h] & ((1u << lane) - 1));  // read only for a nonzero digit
        }
        if (live) {  // the halves side by side (msm_place), one store each for the pair
          const size_t e = (size_t)w * n + 2 * i;  // even (n = 2 scalar_n): 4- and 8-byte aligned stores
          __stcs(reinterpret_cast<uint32_t*>(digits + e), code[0] | code[1] << 16);
          __stcs(reinterpret_cast<uint2*>(ranks + e), make_uint2(rank[0], rank[1]));
        }
      }
    }
  }
}

// Grid (ceil(n / 256), windows): blockIdx.y is the window, so blocks run window by window.
// fixed: every window's digits share the buckets, and the entry names point w * n + i of a
// fixed-base table (2^(c w) P_i at row w). glv: column i holds half i & 1 of scalar i >> 1
// (msm_rank_glv), point (i >> 1) + (i & 1) n / 2.
__global__ void msm_place(const uint16_t* __restrict__ digits, const uint32_t* __restrict__ ranks, size_t n,
                          uint32_t half, int fixed, int glv, const uint32_t* __restrict__ slot_start,
                          uint32_t* __restrict__ sorted) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t w = blockIdx.y;
  const size_t e = (size_t)w * n + i;
  const uint32_t digit = __ldcs(digits + e);
  if (digit == kRankZero) return;
  const uint32_t slot = (fixed ? 0u : w * half) + (digit & 0x7fffu);
  const uint32_t point = fixed ? (uint32_t)e : glv ? (uint32_t)((i >> 1) + (i & 1) * (n >> 1)) : (uint32_t)i;
  sorted[slot_start[slot] + __ldcs(ranks + e)] = point | ((digit & 0x8000u) ? kNegBit : 0u);
}

// Fixed-base table: row w holds 2^(c w) P_i for every base i (affine, Montgomery form, infinity
// as zeros), rows 0..windows-1; an MSM over it needs no per-window buckets and no Horner
// combination. One thread per base: c doublings between rows, one inversion per row.
template <class F>
__global__ void msm_fixed_base_table(const uint32_t* __restrict__ bases, size_t n, uint32_t c, uint32_t windows,
                                     uint32_t* __restrict__ table) {
  constexpr int AW = PointWords<F>::affine;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Xyzz<F> acc = from_affine(load_affine<F>(bases + i * AW));
  for (uint32_t w = 0; w < windows; w++) {
    const Affine<F> a = to_affine(acc);
    uint32_t* o = table + ((size_t)w * n + i) * AW;
    store_elem(o, a.x);
    store_elem(o + AW / 2, a.y);
    if (w + 1 < windows)
      for (uint32_t k = 0; k < c; k++) acc = xyzz_double(acc);
  }
}

// ------------------------------------------------------------------ scan (3 phases)

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total, uint32_t* warp_sums) {
  unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (unsigned)d) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < blockDim.x / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, d);
      if (lane >= (unsigned)d) s += y;
    }
    warp_sums[lane] = s;  // inclusive
  }
  __syncthreads();
  uint32_t before = warp ? warp_sums[warp - 1] : 0;
  *total = warp_sums[blockDim.x / 32 - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanBlock) scan_tile_sums(const uint32_t* __restrict__ in, size_t len,
                                                             uint32_t* __restrict__ tile_sums) {
  __shared__ uint32_t warp_sums[32];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++)
    if (base + k < len) s += in[base + k];
  uint32_t total;
  block_exclusive_scan(s, &total, warp_sums);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Exclusive scan of the tile sums in place (tiles <= kScanTile), total into *grand.
__global__ void __launch_bounds__(kScanBlock) scan_tiles(uint32_t* __restrict__ tile_sums, uint32_t tiles,
                                                          uint32_t* __restrict__ grand) {
  __shared__ uint32_t warp_sums[32];
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint32_t idx = threadIdx.x * kScanItems + k;
    v[k] = idx < tiles ? tile_sums[idx] : 0;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total, warp_sums);
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint32_t idx = threadIdx.x * kScanItems + k;
    if (idx < tiles) tile_sums[idx] = run;
    run += v[k];
  }
  if (threadIdx.x == 0) *grand = total;
}

// out[i] = exclusive prefix of in; also writes it plus out2_bias to out2 (the scatter cursor).
__global__ void __launch_bounds__(kScanBlock) scan_apply(const uint32_t* __restrict__ in, size_t len,
                                                         const uint32_t* __restrict__ tile_offsets,
                                                         uint32_t* __restrict__ out, uint32_t* __restrict__ out2,
                                                         uint32_t out2_bias) {
  __shared__ uint32_t warp_sums[32];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    v[k] = base + k < len ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t total;
  uint32_t run = block_exclusive_scan(s, &total, warp_sums) + tile_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    if (base + k < len) {
      out[base + k] = run;
      out2[base + k] = run + out2_bias;
    }
    run += v[k];
  }
}

// ------------------------------------------------------------------ accumulate

// Largest s in [lo, hi) with a[s] <= p, given a[lo] <= p < a[hi].
__device__ __forceinline__ uint32_t last_leq(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t p) {
  while (hi - lo > 1) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (__ldg(&a[mid]) <= p) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <class F>
__device__ __forceinline__ Affine<F> load_signed_base(const uint32_t* __restrict__ bases, uint32_t entry) {
  Affine<F> p = load_affine<F>(bases + (size_t)(entry & ~kNegBit) * PointWords<F>::affine);
  if (entry & kNegBit) p.y = neg(p.y);
  return p;
}

// One thread per segment [t*L, t*L + L) of the sorted entries (all windows concatenated, slot
// order). slot_start has num_slots + 1 entries; slot_start[num_slots] = total entries.
// Points below `split` come from `bases`, the others from bases2 (point - split): the GLV
// entries' P_i and phi(P_i); plain plans pass split = 2^32 - 1.
template <class F>
__global__ void __launch_bounds__(128) msm_accumulate(const uint32_t* __restrict__ bases,
                                                      const uint32_t* __restrict__ bases2, uint32_t split,
                                                      const uint32_t* __restrict__ sorted,
                                                      const uint32_t* __restrict__ slot_start, uint32_t num_slots,
                                                      uint32_t seg_len, uint32_t* __restrict__ buckets,
                                                      uint32_t* __restrict__ heads,
                                                      uint32_t* __restrict__ head_keys) {
  constexpr int XW = PointWords<F>::xyzz;
  const uint32_t total = __ldg(&slot_start[num_slots]);
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t p0_64 = (uint64_t)t * seg_len;
  if (p0_64 >= total) return;
  const uint32_t p0 = (uint32_t)p0_64;
  const uint64_t e64 = p0_64 + seg_len;
  const uint32_t p1 = e64 < total ? (uint32_t)e64 : total;

  uint32_t s = last_leq(slot_start, 0, num_slots, p0);
  uint32_t end = __ldg(&slot_start[s + 1]);
  bool head = __ldg(&slot_start[s]) < p0;  // the slot began in an earlier segment
  uint32_t head_key = kNoKey;

  Xyzz<F> acc = xyzz_infinity<F>();
  // The next base is fetched into shared memory with cp.async while the current addition runs
  // (two slots per thread), so the prefetch holds no registers.
  constexpr int AW = PointWords<F>::affine;  // 16 (G1) or 32 (G2) words
  __shared__ __align__(16) uint32_t stage[2][128][AW];
  auto stage_base = [&](uint32_t slot, uint32_t e) {
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
    Affine<F> cur = load_affine<F>(&stage[slot][threadIdx.x][0]);
    if (cur_entry & kNegBit) cur.y = neg(cur.y);
    cur_entry = entry;
    slot ^= 1;
    if (p == end) {  // slot s is complete; move to the slot that holds position p
      if (head) {
        store_xyzz(heads + (size_t)t * XW, acc);
        head_key = s;
        head = false;
      } else {
        store_xyzz(buckets + (size_t)s * XW, acc);
      }
      acc = xyzz_infinity<F>();
      uint32_t s2 = s + 1;
      if (__ldg(&slot_start[s2 + 1]) <= p) s2 = last_leq(slot_start, s2, num_slots, p);
      s = s2;
      end = __ldg(&slot_start[s + 1]);
    }
    acc = xyzz_add_affine(acc, cur);
  }
  if (head) {
    store_xyzz(heads + (size_t)t * XW, acc);
    head_key = s;
  } else {
    store_xyzz(buckets + (size_t)s * XW, acc);
  }
  head_keys[t] = head_key;
}

// ------------------------------------------------------------------ merge levels

// Length of the head array at merge level `level` (level 0 = the accumulate output).
__device__ __forceinline__ uint32_t heads_len(uint32_t total, uint32_t seg_len, uint32_t fan_in, uint32_t level) {
  uint64_t len = ((uint64_t)total + seg_len - 1) / seg_len;
  for (uint32_t l = 0; l < level; l++) len = (len + fan_in - 1) / fan_in;
  return (uint32_t)len;
}

template <class F>
__device__ __forceinline__ void add_into_bucket(uint32_t* buckets, uint32_t key, const Xyzz<F>& v) {
  constexpr int XW = PointWords<F>::xyzz;
  uint32_t* b = buckets + (size_t)key * XW;
  store_xyzz(b, xyzz_add(load_xyzz<F>(b), v));
}

// Thread u sums heads [u*f, u*f + f) of a level of len heads (f = fan_in). Runs that start
// inside the range are added into their bucket; a run that continues from the previous range
// becomes this thread's head for the next level. One add per bucket per level (only the range
// where a run starts adds it), so a level needs no atomics.
template <class F>
__device__ __forceinline__ void merge_range(uint32_t u, uint32_t len, uint32_t fan_in, const uint32_t* __restrict__ in_pts,
                                            const uint32_t* __restrict__ in_keys, uint32_t* __restrict__ out_pts,
                                            uint32_t* __restrict__ out_keys, uint32_t* __restrict__ buckets) {
  constexpr int XW = PointWords<F>::xyzz;
  const uint64_t q0_64 = (uint64_t)u * fan_in;
  if (q0_64 >= len) return;
  const uint32_t q0 = (uint32_t)q0_64, q1 = min(q0 + fan_in, len);
  const uint32_t prev = q0 > 0 ? in_keys[q0 - 1] : kNoKey;

  uint32_t cur = kNoKey, start = q0, out_key = kNoKey;
  Xyzz<F> acc = xyzz_infinity<F>();
  for (uint32_t q = q0; q <= q1; q++) {
    uint32_t k = q < q1 ? in_keys[q] : kNoKey;
    if (k != cur || q == q1) {
      if (cur != kNoKey) {
        if (start == q0 && prev == cur) {
          store_xyzz(out_pts + (size_t)u * XW, acc);
          out_key = cur;
        } else {
          add_into_bucket<F>(buckets, cur, acc);
        }
      }
      if (q == q1) break;
      cur = k;
      start = q;
      acc = xyzz_infinity<F>();
    }
    if (k != kNoKey) acc = xyzz_add(acc, load_xyzz<F>(in_pts + (size_t)q * XW));
  }
  out_keys[u] = out_key;
}

// One merge level (grid over its output heads).
template <class F>
__global__ void __launch_bounds__(128) msm_merge(const uint32_t* __restrict__ slot_start, uint32_t num_slots,
                                                 uint32_t seg_len, uint32_t fan_in, uint32_t level,
                                                 const uint32_t* __restrict__ in_pts,
                                                 const uint32_t* __restrict__ in_keys, uint32_t* __restrict__ out_pts,
                                                 uint32_t* __restrict__ out_keys, uint32_t* __restrict__ buckets) {
  const uint32_t total = __ldg(&slot_start[num_slots]);
  const uint32_t len = heads_len(total, seg_len, fan_in, level);
  if (len <= 1) return;  // nothing left to merge
  merge_range<F>(blockIdx.x * blockDim.x + threadIdx.x, len, fan_in, in_pts, in_keys, out_pts, out_keys, buckets);
}

// The last merge levels, from first_level on, in one block of kMergeTailThreads: every such
// level has at most kMergeTailThreads output heads (the host starts the tail where the largest
// possible level fits), the levels run one after another with a block barrier between them
// (the heads of a level are written by the block before the next reads them), and the
// ping-pong buffers alternate by level parity as in msm_merge. The small late levels otherwise
// cost a launch each (about 4-5 us) for a handful of heads.
constexpr uint32_t kMergeTailThreads = 256;
template <class F>
__global__ void __launch_bounds__(kMergeTailThreads) msm_merge_tail(const uint32_t* __restrict__ slot_start,
                                                                   uint32_t num_slots, uint32_t seg_len, uint32_t fan_in,
                                                                   uint32_t first_level, uint32_t levels,
                                                                   uint32_t* __restrict__ heads0,
                                                                   uint32_t* __restrict__ keys0,
                                                                   uint32_t* __restrict__ heads1,
                                                                   uint32_t* __restrict__ keys1,
                                                                   uint32_t* __restrict__ buckets) {
  const uint32_t total = __ldg(&slot_start[num_slots]);
  for (uint32_t l = first_level; l < first_level + levels; l++) {
    const uint32_t len = heads_len(total, seg_len, fan_in, l);
    if (len <= 1) break;  // uniform across the block
    const bool odd = l & 1;
    const uint32_t out_len = (len + fan_in - 1) / fan_in;
    for (uint32_t u = threadIdx.x; u < out_len; u += blockDim.x)
      merge_range<F>(u, len, fan_in, odd ? heads1 : heads0, odd ? keys1 : keys0, odd ? heads0 : heads1,
                     odd ? keys0 : keys1, buckets);
    __syncthreads();
  }
}

// ------------------------------------------------------------------ bucket reduction

// Block-wide sum of XYZZ values (one per thread) through shared memory.
template <class F>
__device__ Xyzz<F> block_sum(Xyzz<F> v, Xyzz<F>* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (unsigned stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride) sh[threadIdx.x] = xyzz_add(sh[threadIdx.x], sh[threadIdx.x + stride]);
    __syncthreads();
  }
  Xyzz<F> r = sh[0];
  __syncthreads();
  return r;
}


// Level of the running-sum reduction. Per window w the input holds m values A_0..A_{m-1} at
// in + (w * in_stride + b) * XW; level 0 reads the buckets, where an empty slot (no entries)
// is the point at infinity. With chunk C = 2^chunk_log, chunk k of window w (b in [Ck, Ck + C)):
//   tot_k = sum_j (j+1) A_{Ck+j},  run_k = sum_j A_{Ck+j} -> run_out[w * run_stride + k - 1] (k >= 1).
// Block (w, j) covers chunks [jT, jT + T) of window w (T = kReduceThreads) and writes the sum of
// their tot_k to tot_out[w * tot_stride + j]: the window-sum stage then reads one point per
// block instead of one per chunk.
template <class F>
__global__ void __launch_bounds__(kReduceThreads) msm_reduce_level(const uint32_t* __restrict__ in, uint32_t in_stride,
                                                                   uint32_t m, uint32_t chunk_log,
                                                                   const uint32_t* __restrict__ slot_start,
                                                                   uint32_t* __restrict__ tot_out, uint32_t tot_stride,
                                                                   uint32_t* __restrict__ run_out, uint32_t run_stride) {
  constexpr int XW = PointWords<F>::xyzz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Xyzz<F>* sh = reinterpret_cast<Xyzz<F>*>(smem_raw);
  const uint32_t chunk = 1u << chunk_log;
  const uint32_t chunks = (m + chunk - 1) / chunk;
  const uint32_t w = blockIdx.y, j = blockIdx.x;
  const uint32_t k = j * kReduceThreads + threadIdx.x;
  Xyzz<F> run = xyzz_infinity<F>(), tot = xyzz_infinity<F>();
  if (k < chunks) {  // no early return: every thread takes part in the block sum below
    const uint32_t lo = k * chunk, hi = min(lo + chunk, m);
    for (uint32_t b = hi; b-- > lo;) {
      size_t slot = (size_t)w * in_stride + b;
      bool empty = slot_start && __ldg(&slot_start[slot]) == __ldg(&slot_start[slot + 1]);
      if (!empty) run = xyzz_add(run, load_xyzz<F>(in + slot * XW));
      tot = xyzz_add(tot, run);
    }
    if (k >= 1) store_xyzz(run_out + ((size_t)w * run_stride + k - 1) * XW, run);
  }
  tot = block_sum(tot, sh);
  if (threadIdx.x == 0) store_xyzz(tot_out + ((size_t)w * tot_stride + j) * XW, tot);
}


// The last level: S = sum_b (b + 1) A_b over m <= kScanLevelMax values per window in one block
// (grid: windows). Thread t owns K = m_pad / 256 consecutive values (K a power of two, at most 4)
// and forms ls_t = sum_j (j + 1) A_{Kt+j} and lt_t = sum_j A_{Kt+j}; then S = sum_t ls_t +
// K sum_{t >= 1} suf_t with suf_t = sum_{u >= t} lt_u, a suffix scan over the threads (Hillis-
// Steele in shared memory) followed by one block sum: about 2K + 2 log2(256) + 2 dependent
// additions, where further chunked levels would each add a chain and a block sum.
template <class F>
__global__ void __launch_bounds__(kScanThreads) msm_reduce_scan(const uint32_t* __restrict__ in, uint32_t in_stride,
                                                                uint32_t m, const uint32_t* __restrict__ slot_start,
                                                                uint32_t* __restrict__ tot_out, uint32_t tot_stride) {
  constexpr int XW = PointWords<F>::xyzz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Xyzz<F>* sh = reinterpret_cast<Xyzz<F>*>(smem_raw);
  const uint32_t w = blockIdx.x, t = threadIdx.x;
  uint32_t k = 1;
  while (k * kScanThreads < m) k <<= 1;
  Xyzz<F> run = xyzz_infinity<F>(), ls = xyzz_infinity<F>();
  for (uint32_t j = k; j-- > 0;) {
    const uint32_t b = t * k + j;
    if (b >= m) continue;
    const size_t slot = (size_t)w * in_stride + b;
    const bool empty = slot_start && __ldg(&slot_start[slot]) == __ldg(&slot_start[slot + 1]);
    if (!empty) run = xyzz_add(run, load_xyzz<F>(in + slot * XW));
    ls = xyzz_add(ls, run);
  }
  // suffix sums of the threads' totals
  Xyzz<F> suf = run;
  sh[t] = suf;
  __syncthreads();
  for (uint32_t d = 1; d < kScanThreads; d <<= 1) {
    const Xyzz<F> other = t + d < kScanThreads ? sh[t + d] : xyzz_infinity<F>();
    __syncthreads();
    suf = xyzz_add(suf, other);
    sh[t] = suf;
    __syncthreads();
  }
  Xyzz<F> next = t + 1 < kScanThreads ? sh[t + 1] : xyzz_infinity<F>();
  __syncthreads();
  for (uint32_t kk = k; kk > 1; kk >>= 1) next = xyzz_double(next);  // K suf_{t+1}
  const Xyzz<F> total = block_sum(xyzz_add(ls, next), sh);
  if (t == 0) store_xyzz(tot_out + (size_t)w * tot_stride * XW, total);
}

// One block per window: S_w = sum over levels l of C^l * sum_k tot_l[k] (C = 2^chunk_log),
// folded from the top level down (chunk_log doublings per level) by warp 0 with lane-parallel
// products.
template <class F>
__global__ void __launch_bounds__(kWindowThreads) msm_window_sums(const uint32_t* __restrict__ tots, ReduceLevels lv,
                                                                  uint32_t* __restrict__ window_sums) {
  constexpr int XW = PointWords<F>::xyzz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Xyzz<F>* sh = reinterpret_cast<Xyzz<F>*>(smem_raw);
  __shared__ uint32_t scratch[32 * 8];
  const LaneScratch sm{scratch};
  const uint32_t w = blockIdx.x;
  Xyzz<F> acc = xyzz_infinity<F>();
  for (int l = (int)lv.count - 1; l >= 0; l--) {
    Xyzz<F> part = xyzz_infinity<F>();
    const uint32_t* base = tots + ((size_t)lv.tot_offset[l] + (size_t)w * lv.tot_len[l]) * XW;
    for (uint32_t k = threadIdx.x; k < lv.tot_len[l]; k += blockDim.x) part = xyzz_add(part, load_xyzz<F>(base + (size_t)k * XW));
    part = block_sum(part, sh);
    if (threadIdx.x < 32) {  // warp 0 folds the levels, products of a level on separate lanes
      for (uint32_t d = 0; d < lv.chunk_log; d++) acc = lane_double(acc, sm);  // x chunk
      acc = lane_add(acc, part, sm);
    }
  }
  if (threadIdx.x == 0) store_xyzz(window_sums + (size_t)w * XW, acc);
}

// result = sum_w 2^(pos_w) S_w by Horner from the top window (msm_combine.wgsl:13-22), by one
// warp: each level's independent products run on separate lanes (curve_lanes.cuh). Window w is
// `base` bits wide, or base + 1 for w < extra (pos_w is the sum of the widths below w): base =
// c, extra = 0 for the plain windows, the glv_window_width split for GLV. F is the
// one-product-per-call form (FqC or Fq2C).
template <class F>
__global__ void __launch_bounds__(32) msm_combine_lanes(const uint32_t* __restrict__ window_sums, uint32_t windows,
                                                        uint32_t base, uint32_t extra, uint32_t* __restrict__ result) {
  __shared__ uint32_t scratch[32 * 8];
  const LaneScratch sm{scratch};
  constexpr int XW = PointWords<F>::xyzz;
  Xyzz<F> acc = load_xyzz<F>(window_sums + (size_t)(windows - 1) * XW);
  for (int w = (int)windows - 2; w >= 0; w--) {
    const uint32_t width = base + ((uint32_t)w < extra ? 1u : 0u);
    for (uint32_t k = 0; k < width; k++) acc = lane_double(acc, sm);
    acc = lane_add(acc, load_xyzz<F>(window_sums + (size_t)w * XW), sm);
  }
  if (threadIdx.x == 0) store_xyzz(result, acc);
}

// result <- result + partial (XYZZ, one thread): the passes of a run over more points than one
// pass holds.
template <class F>
__global__ void msm_add_partial(uint32_t* __restrict__ result, const uint32_t* __restrict__ partial) {
  if (threadIdx.x != 0) return;
  store_xyzz(result, xyzz_add(load_xyzz<F>(result), load_xyzz<F>(partial)));
}

// ------------------------------------------------------------------ base upload

// x <- x * scale / 2^256 for every 8-word Fq coordinate (to_montgomery.wgsl:6-15). With
// scale = 2^512 mod q this maps plain coordinates to Montgomery form; (0,0) stays (0,0).
__global__ void fq_rescale(uint32_t* __restrict__ coords, size_t count, Fq scale) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  store_fe(coords + 8 * i, load_fe<Fq>(coords + 8 * i) * scale);
}

}  // namespace zkg
