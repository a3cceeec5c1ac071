// Fr NTT (src/ntt.rs:1-119, src/shaders/ntt.wgsl, src/shaders/twiddles.wgsl) on sm_100a.
//
// Decimation-in-frequency radix-2, natural order in and out, in place from the caller's view;
// the inverse includes the 1/n factor. Data stays in plain form and twiddles carry the
// Montgomery factor, so a Montgomery product x * tw returns exactly x * w^j (the reference's
// convention, src/ntt.rs:3-5).
//
// The log_n stages run as passes over shared-memory tiles of 2^11 elements (64 KiB; three
// tiles per SM): a pass of s stages loads 2^(11-s) consecutive columns of 2^s rows (rows are
// 2^lm elements apart), so every global access is a run of at least four 32-byte elements.
// The first pass reads the caller's buffer into the plan's scratch, middle passes work in
// place on the scratch, and the last pass writes back in bit-reversed order (fused with the
// 1/n scaling for the inverse). Transforms of at most 2^11 elements are one tile in one block.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "field.cuh"
#include "field_f64.cuh"
#include "host_field.hpp"
#include "ntt.hpp"

namespace zkg {

constexpr uint32_t kTileLog = 11;
constexpr uint32_t kNttThreads = 256;
constexpr uint32_t kMaxStagesPerPass = 9;
// The double-precision form keeps five 8-byte limbs per element in shared memory: tiles of 2^10
// elements (40 KiB) and passes of at most 8 stages keep the same four-element global runs.
constexpr uint32_t kTileLogD = 10;
constexpr uint32_t kMaxStagesPerPassD = 8;

// tw[j] = hi[j >> lo_bits] * lo[j & (2^lo_bits - 1)], j < count (twiddles.wgsl:13-21).
__global__ void ntt_twiddles(const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo, uint32_t lo_bits,
                             size_t count, uint32_t* __restrict__ out) {
  size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  Fr a = load_fe<Fr>(hi + 8 * (j >> lo_bits));
  Fr b = load_fe<Fr>(lo + 8 * (j & ((1ull << lo_bits) - 1)));
  store_fe(out + 8 * j, a * b);
}

__device__ __forceinline__ uint32_t tile_global_index(uint32_t tile, uint32_t slot, uint32_t lg, uint32_t lm,
                                                      uint32_t s) {
  uint32_t row = slot >> lg;
  uint32_t col = slot & ((1u << lg) - 1);
  uint32_t c = (tile << lg) + col;  // column id over the whole array
  uint32_t j0 = c & ((1u << lm) - 1);
  return ((c >> lm) << (lm + s)) + j0 + (row << lm);
}

// One pass: stages [log_n - lm - s, log_n - lm) on tiles of 2^tl elements.
// In the last pass of an inverse, sh_hi / sh_lo (when not null) apply a coset shift: output
// element i (natural order) is multiplied by sh_hi[i >> sh_bits] * sh_lo[i mod 2^sh_bits], the
// low table already holding n^-1 g^j, so the shift replaces the 1/n scaling.
template <bool LAST>
__global__ void __launch_bounds__(kNttThreads, 3)
    ntt_pass(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const uint32_t* __restrict__ tw,
             uint32_t log_n, uint32_t tl, uint32_t lm, uint32_t s, int scale_flag, Fr scale,
             const uint32_t* __restrict__ sh_hi, const uint32_t* __restrict__ sh_lo, uint32_t sh_bits) {
  extern __shared__ __align__(16) uint32_t tile_words[];
  const uint32_t lg = tl - s;
  const uint32_t tile = blockIdx.x;
  const uint32_t elems = 1u << tl;

  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    store_fe(tile_words + 8 * slot, load_fe_cg<Fr>(src + 8 * (size_t)g));
  }
  __syncthreads();

  const uint32_t t0 = log_n - lm - s;  // global index of the pass's first stage
  const uint32_t half_elems = elems >> 1;
  for (uint32_t st = 0; st < s; st++) {
    const uint32_t lh = s - 1 - st;  // log2 of the row distance
    const uint32_t t = t0 + st;      // global stage
    for (uint32_t b = threadIdx.x; b < half_elems; b += kNttThreads) {
      uint32_t col = b & ((1u << lg) - 1);
      uint32_t q = b >> lg;
      uint32_t r_lo = q & ((1u << lh) - 1);
      uint32_t row_a = ((q >> lh) << (lh + 1)) + r_lo;
      uint32_t slot_a = (row_a << lg) + col;
      uint32_t slot_b = slot_a + (1u << (lh + lg));
      uint32_t c = (tile << lg) + col;
      uint32_t j0 = c & ((1u << lm) - 1);
      uint32_t idx = ((r_lo << lm) + j0) << t;
      Fr x = load_fe<Fr>(tile_words + 8 * slot_a);
      Fr y = load_fe<Fr>(tile_words + 8 * slot_b);
      Fr d = x - y;
      store_fe(tile_words + 8 * slot_a, x + y);
      if (idx != 0) d = d * load_fe<Fr>(tw + 8 * (size_t)idx);
      store_fe(tile_words + 8 * slot_b, d);
    }
    __syncthreads();
  }

  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    Fr v = load_fe<Fr>(tile_words + 8 * slot);
    uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    if (LAST) g = __brev(g) >> (32 - log_n);
    if (LAST && sh_hi != nullptr) {
      const Fr gi = load_fe<Fr>(sh_hi + 8 * (size_t)(g >> sh_bits)) *
                    load_fe<Fr>(sh_lo + 8 * (size_t)(g & ((1u << sh_bits) - 1)));
      v = v * gi;
    } else if (scale_flag) {
      v = v * scale;
    }
    store_fe(dst + 8 * (size_t)g, v);
  }
}

// ------------------------------------------------------------------ double-precision form
//
// The same passes with the butterflies in five 52-bit limbs per element (field_f64.cuh;
// Montgomery products issue on the FP64 pipe). Twiddles are held as limbs in Montgomery form
// with R = 2^260, so a product x * tw of a plain x still returns x * w^j. Elements stay below 2r
// in shared memory: x + y is reduced from below 4r, and (x - y + 2r) * tw is below 2r.

__device__ const f64::MultiplesOf<f64::FrLimbs> g_multiples_of_r = f64::MultiplesOf<f64::FrLimbs>();

// Limbs (R = 2^260) of the R = 2^256 Montgomery twiddles, count of them, five doubles each.
__global__ void ntt_twiddles_to_limbs(const uint32_t* __restrict__ tw, size_t count, double* __restrict__ out) {
  size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const Fr a = load_fe<Fr>(tw + 8 * j);
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; i++) w[i] = a.w[i];
  const f64::FqD d = f64::fqd_reduce<f64::FrLimbs>(f64::fqd_from_words_x16(w), &g_multiples_of_r);
#pragma unroll
  for (int k = 0; k < 5; k++) out[5 * j + k] = d.l[k];
}

__device__ __forceinline__ f64::FqD tile_load_d(const double* tile, uint32_t elems, uint32_t slot) {
  return f64::FqD{{tile[slot], tile[elems + slot], tile[2 * elems + slot], tile[3 * elems + slot],
                   tile[4 * elems + slot]}};
}
__device__ __forceinline__ void tile_store_d(double* tile, uint32_t elems, uint32_t slot, const f64::FqD& v) {
#pragma unroll
  for (int k = 0; k < 5; k++) tile[k * elems + slot] = v.l[k];
}

// Canonical words of an element below 2r.
__device__ __forceinline__ Fr fr_from_limbs(const f64::FqD& v) {
  uint32_t w[8];
  f64::limbs_to_words(v.l, w);
  const uint32_t rw[8] = {FrParams::P0, FrParams::P1, FrParams::P2, FrParams::P3,
                          FrParams::P4, FrParams::P5, FrParams::P6, FrParams::P7};
  uint32_t d[8];
  uint32_t borrow = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint64_t t = (uint64_t)w[i] - rw[i] - borrow;
    d[i] = (uint32_t)t;
    borrow = (uint32_t)(t >> 63);
  }
  Fr r;
#pragma unroll
  for (int i = 0; i < 8; i++) r.w[i] = borrow ? w[i] : d[i];
  return r;
}

// ntt_pass with double-precision butterflies; tw holds 5 doubles per twiddle, the tile is stored
// limb-major (limb k of slot e at k * elems + e) so consecutive threads touch consecutive doubles.
// Three blocks of 256 threads per SM (80 registers): with two (116 registers) the warps stalled
// on the twiddle loads (2^24: 5.97 -> 5.32 ms per transform; four blocks spill, 5.40 ms).
// Copying each thread's next-stage twiddles into shared memory with 8-byte cp.async (60 KiB per
// block) made it slower still: 6.49 ms.
template <bool LAST>
__global__ void __launch_bounds__(kNttThreads, 3)
    ntt_pass_f64(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const double* __restrict__ tw,
                 uint32_t log_n, uint32_t tl, uint32_t lm, uint32_t s, int scale_flag, Fr scale_mont,
                 const uint32_t* __restrict__ sh_hi, const uint32_t* __restrict__ sh_lo, uint32_t sh_bits) {
  using namespace f64;
  extern __shared__ __align__(16) double tile_d[];
  const MultiplesOf<FrLimbs>* kr = &g_multiples_of_r;
  const uint32_t lg = tl - s;
  const uint32_t tile = blockIdx.x;
  const uint32_t elems = 1u << tl;

  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    const uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    const Fr v = load_fe_cg<Fr>(src + 8 * (size_t)g);
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = v.w[i];
    FqD d;
    words_to_limbs(w, d.l);
    tile_store_d(tile_d, elems, slot, d);
  }
  __syncthreads();

  const uint32_t t0 = log_n - lm - s;
  const uint32_t half_elems = elems >> 1;
  for (uint32_t st = 0; st < s; st++) {
    const uint32_t lh = s - 1 - st;
    const uint32_t t = t0 + st;
    for (uint32_t b = threadIdx.x; b < half_elems; b += kNttThreads) {
      const uint32_t col = b & ((1u << lg) - 1);
      const uint32_t q = b >> lg;
      const uint32_t r_lo = q & ((1u << lh) - 1);
      const uint32_t row_a = ((q >> lh) << (lh + 1)) + r_lo;
      const uint32_t slot_a = (row_a << lg) + col;
      const uint32_t slot_b = slot_a + (1u << (lh + lg));
      const uint32_t c = (tile << lg) + col;
      const uint32_t j0 = c & ((1u << lm) - 1);
      const uint32_t idx = ((r_lo << lm) + j0) << t;
      const FqD x = tile_load_d(tile_d, elems, slot_a);
      const FqD y = tile_load_d(tile_d, elems, slot_b);
      // Values enter even stages below 2r and odd stages below 4r: an even stage leaves its sums
      // unreduced (below 4r) unless it is the pass's last; an odd stage reduces them (from below
      // 8r). Differences get 4r added in odd stages, so products see inputs below 8r.
      const bool odd = st & 1;
      const FqD sum = fqd_add(x, y);
      tile_store_d(tile_d, elems, slot_a, (odd || st + 1 == s) ? fqd_reduce<FrLimbs>(sum, kr) : sum);
      const FqD d = odd ? fqd_sub<4, FrLimbs>(x, y) : fqd_sub<2, FrLimbs>(x, y);  // (0, 8r)
      FqD out;
      if (idx != 0) {
        const double* w = tw + 5 * (size_t)idx;
        const FqD wd{{__ldg(w), __ldg(w + 1), __ldg(w + 2), __ldg(w + 3), __ldg(w + 4)}};
        out = fqd_mul<FrLimbs>(d, wd);
      } else {
        out = fqd_reduce<FrLimbs>(d, kr);
      }
      tile_store_d(tile_d, elems, slot_b, out);
    }
    __syncthreads();
  }

  const bool shifted = LAST && sh_hi != nullptr;  // the coset shift (with 1/n) as in ntt_pass
  FqD scale;
  if (scale_flag && !shifted) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = scale_mont.w[i];
    scale = fqd_reduce<FrLimbs>(fqd_from_words_x16(w), kr);
  }
  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    FqD v = tile_load_d(tile_d, elems, slot);
    if (scale_flag && !shifted) v = fqd_mul<FrLimbs>(v, scale);
    uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    if (LAST) g = __brev(g) >> (32 - log_n);
    Fr out = fr_from_limbs(v);
    if (shifted) {
      const Fr gi = load_fe<Fr>(sh_hi + 8 * (size_t)(g >> sh_bits)) *
                    load_fe<Fr>(sh_lo + 8 * (size_t)(g & ((1u << sh_bits) - 1)));
      out = out * gi;
    }
    store_fe(dst + 8 * (size_t)g, out);
  }
}

// (a b - c) zinv for plain Fr words, zinv2 = zinv R^2 (the Montgomery form of zinv, times R):
// u = a b / R, w = c / R, (u - w) zinv R^2 / R = (a b - c) zinv.
__device__ __forceinline__ Fr quotient_element(const Fr& a, const Fr& b, const Fr& c, const Fr& zinv2) {
  Fr one = Fr::zero();
  one.w[0] = 1;
  return (a * b - c * one) * zinv2;
}

// ------------------------------------------------------------------ staged-twiddle form
//
// The double-precision butterflies with each stage's twiddles copied into shared memory by
// cp.async during the stage before, from a table laid out in the order the butterflies use
// them. The pass table holds one block of 2^tl entries per distinct tile (a tile's twiddles
// depend on its columns j0 = c mod 2^lm only, so D = 2^max(0, lm - lg) blocks serve all tiles):
// stage st of the pass occupies entries [elems - (elems >> st), elems - (elems >> (st + 1))),
// 2^(lh + lg) twiddles where butterfly b reads entry b mod 2^(lh + lg); each stage block is
// stored limb-major (limb k of entry e at k * size + e), five doubles per twiddle, Montgomery
// form with R = 2^260. The first pass's table is read once per transform (40 bytes per
// element; its tiles share no twiddles), the later passes' tables are small and stay in L2.

// Builds a pass table: entries D * elems, from the seed tables (w^j = hi[j >> lo_bits] * lo[j & mask]).
__global__ void ntt_stage_twiddles(const uint32_t* __restrict__ hi, const uint32_t* __restrict__ lo,
                                   uint32_t lo_bits, uint32_t log_n, uint32_t tl, uint32_t lm, uint32_t s,
                                   size_t entries, double* __restrict__ out) {
  const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= entries) return;
  const uint32_t elems = 1u << tl, lg = tl - s;
  const uint32_t tb = (uint32_t)(id >> tl), off = (uint32_t)(id & (elems - 1));
  const uint32_t v1 = elems - 1 - off;  // stage st holds v1 in [2^(tl-st-1), 2^(tl-st) - 1]
  const uint32_t st = v1 == 0 ? tl : tl - 1 - (31 - __clz(v1));
  double* o = out + (size_t)tb * 5 * elems;
  if (st >= s) {  // padding at the block's end (entries [elems - 2^lg, elems))
#pragma unroll
    for (int k = 0; k < 5; k++) o[5 * (size_t)off + k] = 0.0;
    return;
  }
  const uint32_t base = elems - (elems >> st), size = elems >> (st + 1);
  const uint32_t e = off - base;
  const uint32_t col = e & ((1u << lg) - 1), r_lo = e >> lg;
  const uint32_t c = (tb << lg) + col;
  const uint32_t j0 = c & ((1u << lm) - 1);
  const uint32_t t = log_n - lm - s + st;
  const uint32_t idx = ((r_lo << lm) + j0) << t;  // < n/2
  const Fr w = load_fe<Fr>(hi + 8 * (size_t)(idx >> lo_bits)) * load_fe<Fr>(lo + 8 * (size_t)(idx & ((1u << lo_bits) - 1)));
  uint32_t words[8];
#pragma unroll
  for (int i = 0; i < 8; i++) words[i] = w.w[i];
  const f64::FqD d = f64::fqd_reduce<f64::FrLimbs>(f64::fqd_from_words_x16(words), &g_multiples_of_r);
#pragma unroll
  for (int k = 0; k < 5; k++) o[5 * base + k * size + e] = d.l[k];
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t sa = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}

// Copies stage st's block (5 * size doubles, size = elems >> (st + 1)) into shared memory.
__device__ __forceinline__ void stage_twiddles_async(double* dst, const double* tblock, uint32_t elems, uint32_t st) {
  const uint32_t base = elems - (elems >> st), size = elems >> (st + 1);
  const double* src = tblock + 5 * (size_t)base;
  // 16-byte chunks; a block of one entry (size 1: the last stage of a single-column tile) is
  // copied with the following padding double
  const uint32_t chunks = (5 * size + 1) / 2;
  for (uint32_t i = threadIdx.x; i < chunks; i += blockDim.x) cp_async16(dst + 2 * i, src + 2 * i);
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// A tile of a pass into shared memory as limbs (limb-major), from plain words.
__device__ __forceinline__ void load_tile_f64(const uint32_t* __restrict__ src, double* tile_d, uint32_t tile,
                                              uint32_t lg, uint32_t lm, uint32_t s, uint32_t elems) {
  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    const uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    const Fr v = load_fe_cg<Fr>(src + 8 * (size_t)g);
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = v.w[i];
    f64::FqD d;
    f64::words_to_limbs(w, d.l);
    tile_store_d(tile_d, elems, slot, d);
  }
}

// The pass's output: canonical words, in bit-reversed order in the last pass, with the 1/n
// scaling of an inverse, the fused coset shift (sh_hi != null) or the fused quotient (qa != null).
template <bool LAST>
__device__ __forceinline__ void store_tile_f64(uint32_t* __restrict__ dst, const double* tile_d, uint32_t tile,
                                               uint32_t lg, uint32_t lm, uint32_t s, uint32_t elems, uint32_t log_n,
                                               int scale_flag, const Fr& scale_mont,
                                               const uint32_t* __restrict__ sh_hi, const uint32_t* __restrict__ sh_lo,
                                               uint32_t sh_bits, const uint32_t* __restrict__ qa,
                                               const uint32_t* __restrict__ qb, const Fr& qz2) {
  using namespace f64;
  const MultiplesOf<FrLimbs>* kr = &g_multiples_of_r;
  const bool shifted = LAST && sh_hi != nullptr;
  FqD scale;
  if (scale_flag && !shifted) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = scale_mont.w[i];
    scale = fqd_reduce<FrLimbs>(fqd_from_words_x16(w), kr);
  }
  for (uint32_t slot = threadIdx.x; slot < elems; slot += kNttThreads) {
    FqD v = tile_load_d(tile_d, elems, slot);
    if (scale_flag && !shifted) v = fqd_mul<FrLimbs>(v, scale);
    uint32_t g = tile_global_index(tile, slot, lg, lm, s);
    if (LAST) g = __brev(g) >> (32 - log_n);
    Fr out = fr_from_limbs(v);
    if (shifted) {
      const Fr gi = load_fe<Fr>(sh_hi + 8 * (size_t)(g >> sh_bits)) *
                    load_fe<Fr>(sh_lo + 8 * (size_t)(g & ((1u << sh_bits) - 1)));
      out = out * gi;
    }
    if (LAST && qa != nullptr)
      out = quotient_element(load_fe<Fr>(qa + 8 * (size_t)g), load_fe<Fr>(qb + 8 * (size_t)g), out, qz2);
    store_fe(dst + 8 * (size_t)g, out);
  }
}

// One pass as ntt_pass_f64, with staged twiddles (tw: this pass's table, tw_mask = D - 1).
// Shared memory: the tile (5 * elems doubles) and two twiddle buffers (stage 0, 2, ...: elems/2
// entries; stage 1, 3, ...: elems/4), 70 KiB for tiles of 2^10 elements.
template <bool LAST, bool PAIR>
__global__ void __launch_bounds__(kNttThreads, PAIR ? 2 : 3)
    ntt_pass_f64s(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const double* __restrict__ tw,
                  uint32_t tw_mask, uint32_t log_n, uint32_t tl, uint32_t lm, uint32_t s, int scale_flag,
                  Fr scale_mont, const uint32_t* __restrict__ sh_hi, const uint32_t* __restrict__ sh_lo,
                  uint32_t sh_bits, const uint32_t* __restrict__ qa, const uint32_t* __restrict__ qb, Fr qz2) {
  using namespace f64;
  extern __shared__ __align__(16) double smem_d[];
  const MultiplesOf<FrLimbs>* kr = &g_multiples_of_r;
  const uint32_t lg = tl - s;
  const uint32_t tile = blockIdx.x;
  const uint32_t elems = 1u << tl;
  double* tile_d = smem_d;
  double* const twbuf0 = smem_d + 5 * elems;                   // stages 0, 2, 4, ...
  double* const twbuf1 = smem_d + 5 * elems + 5 * (elems >> 1);  // stages 1, 3, 5, ...
  const double* tblock = tw + (size_t)(tile & tw_mask) * 5 * elems;

  stage_twiddles_async(twbuf0, tblock, elems, 0);
  load_tile_f64(src, tile_d, tile, lg, lm, s, elems);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();

  const uint32_t half_elems = elems >> 1;
  for (uint32_t st = 0; st < s; st++) {
    if (st + 1 < s) stage_twiddles_async((st & 1) ? twbuf0 : twbuf1, tblock, elems, st + 1);
    const uint32_t lh = s - 1 - st;
    const uint32_t size = elems >> (st + 1);  // = 2^(lh + lg)
    const double* twst = (st & 1) ? twbuf1 : twbuf0;
    if (PAIR && half_elems % (2 * kNttThreads) == 0) {
      // two butterflies per iteration, loads first: two independent products in flight
      for (uint32_t b0 = threadIdx.x; b0 < half_elems; b0 += 2 * kNttThreads) {
        uint32_t sa[2], sb[2];
        FqD x[2], y[2], w[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
          const uint32_t b = b0 + k * kNttThreads;
          const uint32_t col = b & ((1u << lg) - 1);
          const uint32_t q = b >> lg;
          const uint32_t r_lo = q & ((1u << lh) - 1);
          const uint32_t row_a = ((q >> lh) << (lh + 1)) + r_lo;
          sa[k] = (row_a << lg) + col;
          sb[k] = sa[k] + (1u << (lh + lg));
          const uint32_t j0 = ((tile << lg) + col) & ((1u << lm) - 1);
          const uint32_t e = b & (size - 1);
          w[k] = (r_lo | j0) != 0
                     ? FqD{{twst[e], twst[size + e], twst[2 * size + e], twst[3 * size + e], twst[4 * size + e]}}
                     : frd_one260();  // a product by one in Montgomery form returns the value, below 2r
          x[k] = tile_load_d(tile_d, elems, sa[k]);
          y[k] = tile_load_d(tile_d, elems, sb[k]);
        }
        const FqD s0 = fqd_reduce<FrLimbs>(fqd_add(x[0], y[0]), kr);
        const FqD s1 = fqd_reduce<FrLimbs>(fqd_add(x[1], y[1]), kr);
        const FqD o0 = fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x[0], y[0]), w[0]);
        const FqD o1 = fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x[1], y[1]), w[1]);
        tile_store_d(tile_d, elems, sa[0], s0);
        tile_store_d(tile_d, elems, sa[1], s1);
        tile_store_d(tile_d, elems, sb[0], o0);
        tile_store_d(tile_d, elems, sb[1], o1);
      }
    } else
    for (uint32_t b = threadIdx.x; b < half_elems; b += kNttThreads) {
      const uint32_t col = b & ((1u << lg) - 1);
      const uint32_t q = b >> lg;
      const uint32_t r_lo = q & ((1u << lh) - 1);
      const uint32_t row_a = ((q >> lh) << (lh + 1)) + r_lo;
      const uint32_t slot_a = (row_a << lg) + col;
      const uint32_t slot_b = slot_a + (1u << (lh + lg));
      const uint32_t c = (tile << lg) + col;
      const uint32_t j0 = c & ((1u << lm) - 1);
      const FqD x = tile_load_d(tile_d, elems, slot_a);
      const FqD y = tile_load_d(tile_d, elems, slot_b);
      // Values enter even stages below 2r and odd stages below 4r: an even stage leaves its sums
      // unreduced (below 4r) unless it is the pass's last; an odd stage reduces them (from below
      // 8r). Differences get 4r added in odd stages, so products see inputs below 8r.
      const bool odd = st & 1;
      const FqD sum = fqd_add(x, y);
      tile_store_d(tile_d, elems, slot_a, (odd || st + 1 == s) ? fqd_reduce<FrLimbs>(sum, kr) : sum);
      const FqD d = odd ? fqd_sub<4, FrLimbs>(x, y) : fqd_sub<2, FrLimbs>(x, y);  // (0, 8r)
      FqD out;
      if ((r_lo | j0) != 0) {
        const uint32_t e = b & (size - 1);
        const FqD wd{{twst[e], twst[size + e], twst[2 * size + e], twst[3 * size + e], twst[4 * size + e]}};
        out = fqd_mul<FrLimbs>(d, wd);
      } else {
        out = fqd_reduce<FrLimbs>(d, kr);
      }
      tile_store_d(tile_d, elems, slot_b, out);
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }

  store_tile_f64<LAST>(dst, tile_d, tile, lg, lm, s, elems, log_n, scale_flag, scale_mont, sh_hi, sh_lo, sh_bits, qa,
                       qb, qz2);
}

// Radix-4 form (form 4): the stages of a pass two at a time. A thread takes rows r0, r0 + h/2,
// r0 + h, r0 + 3h/2 of one column (h = 2^lh the first stage's row distance): the first stage's
// two butterflies (r0, r0 + h) and (r0 + h/2, r0 + 3h/2), then the second stage's (r0, r0 + h/2)
// and (r0 + h, r0 + 3h/2), which share one twiddle: four products and three twiddles per four
// elements, as in two radix-2 stages, with half the shared-memory round trips and barriers. An
// odd last stage runs as radix-2. Twiddle buffers: two sets, each holding the blocks of one step
// (stages 0 and 1: 3/4 of a tile's entries; stages 2 and 3: 3/16), the next step's copied in
// while the current one runs. Shared memory: 40 + 37.5 KiB for tiles of 2^10 elements.
template <bool LAST>
__global__ void __launch_bounds__(kNttThreads, 2)
    ntt_pass_f64r4(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const double* __restrict__ tw,
                   uint32_t tw_mask, uint32_t log_n, uint32_t tl, uint32_t lm, uint32_t s, int scale_flag,
                   Fr scale_mont, const uint32_t* __restrict__ sh_hi, const uint32_t* __restrict__ sh_lo,
                   uint32_t sh_bits, const uint32_t* __restrict__ qa, const uint32_t* __restrict__ qb, Fr qz2) {
  using namespace f64;
  extern __shared__ __align__(16) double smem_d[];
  const MultiplesOf<FrLimbs>* kr = &g_multiples_of_r;
  const uint32_t lg = tl - s;
  const uint32_t tile = blockIdx.x;
  const uint32_t elems = 1u << tl;
  double* tile_d = smem_d;
  // set 0: steps 0, 2, ... (first step: stage 0 block of elems/2 entries, stage 1 of elems/4);
  // set 1: steps 1, 3, ... (stage 2: elems/8, stage 3: elems/16). 5 doubles per entry.
  double* const set0 = smem_d + 5 * elems;
  double* const set1 = set0 + 5 * ((elems >> 1) + (elems >> 2));
  const double* tblock = tw + (size_t)(tile & tw_mask) * 5 * elems;
  auto copy_step = [&](double* set, uint32_t st) {  // blocks of stages st and st + 1 (when it exists)
    stage_twiddles_async(set, tblock, elems, st);
    if (st + 1 < s) stage_twiddles_async(set + 5 * (elems >> (st + 1)), tblock, elems, st + 1);
  };

  copy_step(set0, 0);
  load_tile_f64(src, tile_d, tile, lg, lm, s, elems);
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();

  const FqD one = frd_one260();
  for (uint32_t st = 0, step = 0; st < s; st += 2, step++) {
    if (st + 2 < s) copy_step((step & 1) ? set0 : set1, st + 2);
    const double* twa = (step & 1) ? set1 : set0;
    const uint32_t lh = s - 1 - st;
    const uint32_t size_a = elems >> (st + 1);  // = 2^(lh + lg)
    if (st + 1 < s) {
      const double* twb = twa + 5 * size_a;
      const uint32_t size_b = size_a >> 1;
      const uint32_t hh = 1u << (lh - 1);
      for (uint32_t u = threadIdx.x; u < (elems >> 2); u += kNttThreads) {
        const uint32_t col = u & ((1u << lg) - 1);
        const uint32_t q4 = u >> lg;
        const uint32_t rr = q4 & (hh - 1);
        const uint32_t r0 = ((q4 >> (lh - 1)) << (lh + 1)) + rr;
        const uint32_t j0 = ((tile << lg) + col) & ((1u << lm) - 1);
        const uint32_t s0 = (r0 << lg) + col, s1 = s0 + (hh << lg), s2 = s0 + (2 * hh << lg),
                       s3 = s0 + (3 * hh << lg);
        const uint32_t e0 = (rr << lg) + col, e1 = ((rr + hh) << lg) + col;
        const bool unit = (rr | j0) == 0;  // twiddle 1 for the first butterfly of each stage
        // Bounds: tile values below 2r. The first stage's sums stay unreduced (below 4r): the
        // second stage reduces their sum (below 8r) and multiplies their difference (plus 4r,
        // below 8r), both within what fqd_reduce (16r) and the product (below 2r out) take.
        const FqD x0 = tile_load_d(tile_d, elems, s0), x2 = tile_load_d(tile_d, elems, s2);
        const FqD wa0 = unit ? one : FqD{{twa[e0], twa[size_a + e0], twa[2 * size_a + e0], twa[3 * size_a + e0], twa[4 * size_a + e0]}};
        const FqD y0 = fqd_add(x0, x2);
        const FqD y2 = fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x0, x2), wa0);
        const FqD x1 = tile_load_d(tile_d, elems, s1), x3 = tile_load_d(tile_d, elems, s3);
        const FqD wa1{{twa[e1], twa[size_a + e1], twa[2 * size_a + e1], twa[3 * size_a + e1], twa[4 * size_a + e1]}};
        const FqD y1 = fqd_add(x1, x3);
        const FqD y3 = fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x1, x3), wa1);
        const FqD wb = unit ? one : FqD{{twb[e0], twb[size_b + e0], twb[2 * size_b + e0], twb[3 * size_b + e0], twb[4 * size_b + e0]}};
        tile_store_d(tile_d, elems, s0, fqd_reduce<FrLimbs>(fqd_add(y0, y1), kr));
        tile_store_d(tile_d, elems, s1, fqd_mul<FrLimbs>(fqd_sub<4, FrLimbs>(y0, y1), wb));
        tile_store_d(tile_d, elems, s2, fqd_reduce<FrLimbs>(fqd_add(y2, y3), kr));
        tile_store_d(tile_d, elems, s3, fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(y2, y3), wb));
      }
    } else {  // one stage left (lh = 0): radix-2 butterflies of rows (2i, 2i + 1)
      for (uint32_t b = threadIdx.x; b < (elems >> 1); b += kNttThreads) {
        const uint32_t col = b & ((1u << lg) - 1);
        const uint32_t q = b >> lg;
        const uint32_t slot_a = ((2 * q) << lg) + col, slot_b = slot_a + (1u << lg);
        const uint32_t j0 = ((tile << lg) + col) & ((1u << lm) - 1);
        const uint32_t e = b & (size_a - 1);
        const FqD w = j0 == 0 ? one : FqD{{twa[e], twa[size_a + e], twa[2 * size_a + e], twa[3 * size_a + e], twa[4 * size_a + e]}};
        const FqD x = tile_load_d(tile_d, elems, slot_a), y = tile_load_d(tile_d, elems, slot_b);
        tile_store_d(tile_d, elems, slot_a, fqd_reduce<FrLimbs>(fqd_add(x, y), kr));
        tile_store_d(tile_d, elems, slot_b, fqd_mul<FrLimbs>(fqd_sub<2, FrLimbs>(x, y), w));
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
  store_tile_f64<LAST>(dst, tile_d, tile, lg, lm, s, elems, log_n, scale_flag, scale_mont, sh_hi, sh_lo, sh_bits, qa,
                       qb, qz2);
}

static std::vector<uint32_t> powers_words(const host::U256& step, size_t len) {
  const host::Field& f = host::fr();
  std::vector<uint32_t> out(8 * len);
  host::U256 x = f.one;  // Montgomery 1
  for (size_t i = 0; i < len; i++) {
    host::words32(x, &out[8 * i]);
    x = host::mul(x, step, f);
  }
  return out;
}

// The largest dynamic shared memory a pass launch asks for (a function attribute: one value for
// every plan on the device, so always the largest tile's; the double-precision tiles, 40 KiB,
// stay under the 48 KiB that needs no attribute).
static void set_pass_smem_limits() {
  const int smem = (int)((size_t)32 << kTileLog);
  check_cuda(cudaFuncSetAttribute(ntt_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
             "ntt smem attribute");
  check_cuda(cudaFuncSetAttribute(ntt_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
             "ntt smem attribute");
  const int smem_s = (int)((size_t)70 << kTileLogD);  // tile + two twiddle buffers, forms 2 and 3
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64s<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_s),
             "ntt smem attribute");
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64s<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_s),
             "ntt smem attribute");
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64s<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_s),
             "ntt smem attribute");
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64s<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_s),
             "ntt smem attribute");
  const int smem_r4 = (int)((size_t)80 << kTileLogD);  // tile + two step buffer sets, form 4
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64r4<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_r4),
             "ntt smem attribute");
  check_cuda(cudaFuncSetAttribute(ntt_pass_f64r4<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_r4),
             "ntt smem attribute");
}

NttPlan::NttPlan(zkg_ctx* c, uint32_t log_n_) : ctx(c), log_n(log_n_) {
  if (log_n < 10 || log_n > 27) fail(ZKG_EINVAL, "log_n must be in 10..=27");
  use(ctx);
  const host::Field& f = host::fr();
  const size_t n = (size_t)1 << log_n;
  host::U256 w = host::root_of_unity(log_n);  // Montgomery form
  host::U256 w_inv = host::inverse(w, f);
  // n^-1 * R (src/ntt.rs:32): Montgomery form of 1/n
  host::U256 n_inv = host::inverse(host::to_mont(host::U256{{(uint64_t)n, 0, 0, 0}}, f), f);
  host::words32(n_inv, n_inv_words);

  scratch.alloc(8 * n, "ntt scratch");
  build_seeds(w, seeds[0]);
  build_seeds(w_inv, seeds[1]);
  set_pass_smem_limits();
  // Double-precision butterflies with staged twiddles by default, two per thread step up to 2^17
  // elements: measured on B200 (ms per transform) 2^16: form 3 0.048, form 2 0.050, form 1
  // 0.054, form 0 0.089; 2^20: form 2 0.292, form 3 0.302, form 1 0.313; 2^24: form 2 5.00,
  // form 3 5.30, forms 0 and 1 5.33.
  set_variant(log_n <= 17 ? 3 : 2);
}

uint32_t NttPlan::tile_log() const { return variant != 0 ? kTileLogD : kTileLog; }

bool NttPlan::set_variant(int v) {
  if (v < 0 || v > 4) return false;
  if (v <= 1 && !fwd_tw.ptr) {  // the table of w^j on first use of a form that reads it
    use(ctx);
    build_twiddles(seeds[0], fwd_tw);
    build_twiddles(seeds[1], inv_tw);
    check_cuda(cudaStreamSynchronize(ctx->setup), "ntt twiddles");
  }
  if (v == 1 && !fwd_twd.ptr) {  // twiddle limbs on first use of the double-precision form
    const size_t count = (size_t)1 << (log_n - 1);
    use(ctx);
    fwd_twd.alloc(10 * count, "ntt twiddle limbs");
    inv_twd.alloc(10 * count, "ntt twiddle limbs");
    ntt_twiddles_to_limbs<<<grid_for(count, 256), 256, 0, ctx->setup>>>(fwd_tw.ptr, count,
                                                                        reinterpret_cast<double*>(fwd_twd.ptr));
    check_launch("ntt_twiddles_to_limbs");
    ntt_twiddles_to_limbs<<<grid_for(count, 256), 256, 0, ctx->setup>>>(inv_tw.ptr, count,
                                                                        reinterpret_cast<double*>(inv_twd.ptr));
    check_launch("ntt_twiddles_to_limbs");
    check_cuda(cudaStreamSynchronize(ctx->setup), "ntt twiddle limbs");
  }
  variant = v;
  // Pass split: one tile when it fits, else passes of near-equal size, at most 9 stages each
  // (integer form, tiles of 2^11) or 8 (double-precision forms, tiles of 2^10).
  set_max_stages(v != 0 ? kMaxStagesPerPassD : kMaxStagesPerPass);
  return true;
}

bool NttPlan::set_max_stages(uint32_t ms) {
  const uint32_t tlog = tile_log();
  const uint32_t def = variant != 0 ? kMaxStagesPerPassD : kMaxStagesPerPass;
  if (ms < 6 || ms > tlog) return false;
  bool ok = true;
  if (log_n <= tlog) {
    passes.assign(1, log_n);
    max_stages = def;
    ok = ms == def;
  } else {
    max_stages = ms;
    uint32_t p = (log_n + ms - 1) / ms;
    passes.clear();
    for (uint32_t i = 0; i < p; i++) passes.push_back(log_n / p + (i < log_n % p ? 1u : 0u));
  }
  if (variant >= 2) build_stage_tables();
  return ok;
}

void NttPlan::build_stage_tables() {
  use(ctx);
  const uint32_t tl = log_n < kTileLogD ? log_n : kTileLogD;
  const uint32_t lo_bits = log_n / 2;  // as build_twiddles: ceil((log_n - 1) / 2)
  for (int dir = 0; dir < 2; dir++) stage_tw[dir].clear();
  stage_tw_mask.clear();
  uint32_t done = 0;
  for (uint32_t st : passes) {
    const uint32_t lm = log_n - done - st;
    const int spare = (int)log_n - (int)done - (int)tl;  // log2 of the distinct tile blocks
    const size_t blocks = (size_t)1 << (spare > 0 ? spare : 0);
    const size_t entries = blocks << tl;
    stage_tw_mask.push_back((uint32_t)(blocks - 1));
    for (int dir = 0; dir < 2; dir++) {
      std::unique_ptr<DeviceArray> t(new DeviceArray);
      t->alloc(10 * entries, "ntt staged twiddles");
      ntt_stage_twiddles<<<grid_for(entries, 256), 256, 0, ctx->setup>>>(
          seeds[dir][1].ptr, seeds[dir][0].ptr, lo_bits, log_n, tl, lm, st, entries, t->as<double>());
      check_launch("ntt_stage_twiddles");
      stage_tw[dir].push_back(std::move(t));
    }
    done += st;
  }
  check_cuda(cudaStreamSynchronize(ctx->setup), "ntt staged twiddles");
}

// Seed tables of one direction: lo[j] = w^j (j < 2^lo_bits) and hi[k] = w^(k 2^lo_bits), so
// that w^j = hi[j >> lo_bits] * lo[j mod 2^lo_bits] for j < n/2 (twiddles.wgsl:13-21).
void NttPlan::build_seeds(const host::U256& root, DeviceArray (&seed)[2]) {
  const host::Field& f = host::fr();
  const size_t count = (size_t)1 << (log_n - 1);
  const uint32_t lo_bits = (log_n - 1 + 1) / 2;  // ceil((log_n - 1) / 2)
  const size_t lo_len = (size_t)1 << lo_bits;
  const size_t hi_len = (count + lo_len - 1) / lo_len;
  std::vector<uint32_t> lo = powers_words(root, lo_len);
  host::U256 step = host::pow(root, host::U256{{(uint64_t)lo_len, 0, 0, 0}}, f);
  std::vector<uint32_t> hi = powers_words(step, hi_len);
  DeviceArray& dlo = seed[0];
  DeviceArray& dhi = seed[1];
  dlo.alloc(lo.size(), "ntt twiddle seeds");
  dhi.alloc(hi.size(), "ntt twiddle seeds");
  // From pageable host memory: the call returns once the host vectors have been staged.
  check_cuda(cudaMemcpyAsync(dlo.ptr, lo.data(), lo.size() * 4, cudaMemcpyHostToDevice, ctx->setup), "twiddle copy");
  check_cuda(cudaMemcpyAsync(dhi.ptr, hi.data(), hi.size() * 4, cudaMemcpyHostToDevice, ctx->setup), "twiddle copy");
}

// The table of w^j, j < n/2, from a direction's seeds (set-up stream).
void NttPlan::build_twiddles(DeviceArray (&seed)[2], DeviceArray& out) {
  const size_t count = (size_t)1 << (log_n - 1);
  const uint32_t lo_bits = (log_n - 1 + 1) / 2;
  out.alloc(8 * count, "ntt twiddles");
  ntt_twiddles<<<grid_for(count, 256), 256, 0, ctx->setup>>>(seed[1].ptr, seed[0].ptr, lo_bits, count, out.ptr);
  check_launch("ntt_twiddles");
}

// lo'[j] = lo[j] * f (Montgomery products), j < len.
__global__ void scale_powers_kernel(const uint32_t* __restrict__ lo, size_t len, Fr f, uint32_t* __restrict__ out) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= len) return;
  store_fe(out + 8 * j, load_fe<Fr>(lo + 8 * j) * f);
}

const NttPlan::FusedShift* NttPlan::fused_for(const CosetShift& shift) {
  for (auto& f : fused)
    if (f->serial == shift.serial) return f.get();
  if (shift.log_n != log_n)
    fail(ZKG_EINVAL, "coset shift of 2^" + std::to_string(shift.log_n) + " elements on a 2^" + std::to_string(log_n) +
                         " transform");
  std::unique_ptr<FusedShift> f(new FusedShift);
  f->serial = shift.serial;
  const size_t len = (size_t)1 << shift.lo_bits;
  f->lo.alloc(8 * len, "fused coset table");
  Fr inv_n;
  std::memcpy(inv_n.w, n_inv_words, sizeof(inv_n.w));
  use(ctx);
  scale_powers_kernel<<<grid_for(len, 256), 256, 0, ctx->setup>>>(shift.lo.ptr, len, inv_n, f->lo.ptr);
  check_launch("scale_powers_kernel");
  // Set-up work runs on the set-up stream: done before the plan uses the table on any stream.
  check_cuda(cudaStreamSynchronize(ctx->setup), "fused coset table");
  fused.push_back(std::move(f));
  return fused.back().get();
}

void NttPlan::prepare_shift(const CosetShift& shift) { fused_for(shift); }

void NttPlan::enqueue(uint32_t* data, bool inverse, cudaStream_t s, const CosetShift* shift, const Quotient* quot) {
  if (shift && !inverse) fail(ZKG_EINVAL, "a fused coset shift follows an inverse transform");
  if (quot && inverse) fail(ZKG_EINVAL, "a fused quotient follows a forward transform");
  if (quot && variant < 2) {  // forms without the fused epilogue: the transform, then the kernel
    enqueue(data, false, s);
    quotient(data, quot->a, quot->b, data, log_n, quot->zinv, s);
    return;
  }
  const uint32_t* qa = quot ? quot->a : nullptr;
  const uint32_t* qb = quot ? quot->b : nullptr;
  Fr qz2;
  if (quot) {
    const host::Field& f = host::fr();
    host::words32(host::to_mont(host::to_mont(quot->zinv, f), f), qz2.w);
  }
  const FusedShift* fs = shift ? fused_for(*shift) : nullptr;
  const uint32_t* sh_hi = fs ? shift->hi.ptr : nullptr;
  const uint32_t* sh_lo = fs ? fs->lo.ptr : nullptr;
  const uint32_t sh_bits = fs ? shift->lo_bits : 0;
  const uint32_t* tw = inverse ? inv_tw.ptr : fwd_tw.ptr;
  const double* twd = reinterpret_cast<const double*>(inverse ? inv_twd.ptr : fwd_twd.ptr);
  Fr scale;
  std::memcpy(scale.w, n_inv_words, sizeof(scale.w));
  const uint32_t tlog = tile_log();
  const uint32_t tl = log_n < tlog ? log_n : tlog;
  const unsigned tiles = 1u << (log_n - tl);
  const size_t smem = variant == 4   ? (size_t)80 << tl
                      : variant >= 2 ? (size_t)70 << tl
                      : variant == 1 ? (size_t)40 << tl
                                     : (size_t)32 << tl;
  uint32_t done = 0;
  const size_t np = passes.size();
  for (size_t i = 0; i < np; i++) {
    const uint32_t st = passes[i];
    const uint32_t lm = log_n - done - st;
    const bool last = i + 1 == np;
    const uint32_t* src = i == 0 ? data : scratch.ptr;
    uint32_t* dst = last ? data : scratch.ptr;
    const int scale_flag = last && inverse;
    size_t ev = timer.enabled ? timer.begin((int)i, s) : 0;
    const double* stw = variant >= 2 ? stage_tw[inverse ? 1 : 0][i]->as<double>() : nullptr;
    if (variant == 4 && last)
      ntt_pass_f64r4<true><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm, st,
                                                            scale_flag, scale, sh_hi, sh_lo, sh_bits, qa, qb, qz2);
    else if (variant == 4)
      ntt_pass_f64r4<false><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm, st,
                                                             scale_flag, scale, nullptr, nullptr, 0, nullptr, nullptr,
                                                             qz2);
    else if (variant == 2 && last)
      ntt_pass_f64s<true, false><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm,
                                                                  st, scale_flag, scale, sh_hi, sh_lo, sh_bits, qa, qb, qz2);
    else if (variant == 2)
      ntt_pass_f64s<false, false><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm,
                                                                   st, scale_flag, scale, nullptr, nullptr, 0, nullptr, nullptr, qz2);
    else if (variant == 3 && last)
      ntt_pass_f64s<true, true><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm,
                                                                 st, scale_flag, scale, sh_hi, sh_lo, sh_bits, qa, qb, qz2);
    else if (variant == 3)
      ntt_pass_f64s<false, true><<<tiles, kNttThreads, smem, s>>>(src, dst, stw, stage_tw_mask[i], log_n, tl, lm,
                                                                  st, scale_flag, scale, nullptr, nullptr, 0, nullptr,
                                                                  nullptr, qz2);
    else if (variant == 1 && last)
      ntt_pass_f64<true><<<tiles, kNttThreads, smem, s>>>(src, dst, twd, log_n, tl, lm, st, scale_flag, scale, sh_hi,
                                                          sh_lo, sh_bits);
    else if (variant == 1)
      ntt_pass_f64<false><<<tiles, kNttThreads, smem, s>>>(src, dst, twd, log_n, tl, lm, st, scale_flag, scale,
                                                           nullptr, nullptr, 0);
    else if (last)
      ntt_pass<true><<<tiles, kNttThreads, smem, s>>>(src, dst, tw, log_n, tl, lm, st, scale_flag, scale, sh_hi,
                                                      sh_lo, sh_bits);
    else
      ntt_pass<false><<<tiles, kNttThreads, smem, s>>>(src, dst, tw, log_n, tl, lm, st, scale_flag, scale, nullptr,
                                                       nullptr, 0);
    check_launch("ntt_pass");
    if (timer.enabled) timer.end(ev, s);
    done += st;
  }
  if (timer.enabled) timer.runs++;
}

void NttPlan::run(zkg_buf* data, bool inverse, const CosetShift* shift, const Quotient* quot) {
  const size_t need = (size_t)32 << log_n;
  const size_t have = data->words * 4;
  if (have < need)
    fail(ZKG_ESIZE, "data buffer holds " + std::to_string(have) + " bytes; a 2^" + std::to_string(log_n) +
                        " transform needs " + std::to_string(need));
  use(ctx);
  enqueue(data->ptr, inverse, ctx->stream, shift, quot);
}

}  // namespace zkg

namespace zkg {

// ------------------------------------------------------------------ coset shift
//
// x_i <- x_i * g^i for i < n (the distribute-powers step between the inverse and forward
// transforms of a Groth16 witness map; README.md:229-230 of the reference names it as a kernel
// on top). g^i = hi[i >> lo_bits] * lo[i & mask] from two small tables of powers, so
// each element costs two Fr products and one read and write of 32 bytes.
__global__ void coset_shift_kernel(uint32_t* __restrict__ data, size_t n, const uint32_t* __restrict__ hi,
                                   const uint32_t* __restrict__ lo, uint32_t lo_bits) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Fr p = load_fe<Fr>(hi + 8 * (i >> lo_bits)) * load_fe<Fr>(lo + 8 * (i & ((1ull << lo_bits) - 1)));
  store_fe(data + 8 * i, load_fe<Fr>(data + 8 * i) * p);
}

static std::atomic<uint64_t> g_coset_serial{1};

CosetShift::CosetShift(zkg_ctx* c, uint32_t log_n_, const uint32_t* g_plain)
    : ctx(c), log_n(log_n_), serial(g_coset_serial.fetch_add(1)) {
  if (log_n < 1 || log_n > 28) fail(ZKG_EINVAL, "log_n must be in 1..=28");
  use(ctx);
  const host::Field& f = host::fr();
  const host::U256 g_raw = host::from_words32(g_plain);
  if (!(host::geq(f.p, g_raw) && !host::eq(f.p, g_raw))) fail(ZKG_EINVAL, "coset generator must be below r");
  host::U256 g = host::to_mont(g_raw, f);
  const size_t n = (size_t)1 << log_n;
  lo_bits = (log_n + 1) / 2;
  const size_t lo_len = (size_t)1 << lo_bits;
  const size_t hi_len = (n + lo_len - 1) / lo_len;
  std::vector<uint32_t> lo_h = powers_words(g, lo_len);
  std::vector<uint32_t> hi_h = powers_words(host::pow(g, host::U256{{(uint64_t)lo_len, 0, 0, 0}}, f), hi_len);
  lo.alloc(lo_h.size(), "coset powers");
  hi.alloc(hi_h.size(), "coset powers");
  check_cuda(cudaMemcpyAsync(lo.ptr, lo_h.data(), lo_h.size() * 4, cudaMemcpyHostToDevice, ctx->setup), "copy");
  check_cuda(cudaMemcpyAsync(hi.ptr, hi_h.data(), hi_h.size() * 4, cudaMemcpyHostToDevice, ctx->setup), "copy");
  // Set-up work runs on the set-up stream: done before the shift is used on any stream.
  check_cuda(cudaStreamSynchronize(ctx->setup), "coset powers");
}

void CosetShift::enqueue(uint32_t* data, cudaStream_t s) {
  const size_t n = (size_t)1 << log_n;
  coset_shift_kernel<<<grid_for(n, 256), 256, 0, s>>>(data, n, hi.ptr, lo.ptr, lo_bits);
  check_launch("coset_shift_kernel");
}

void CosetShift::run(zkg_buf* data) {
  const size_t need = (size_t)8 << log_n;
  if (data->words < need)
    fail(ZKG_ESIZE, "data buffer holds " + std::to_string(data->words * 4) + " bytes; a coset shift of 2^" +
                        std::to_string(log_n) + " elements needs " + std::to_string(need * 4));
  use(ctx);
  enqueue(data->ptr, ctx->stream);
}

// ------------------------------------------------------------------ quotient on the coset
//
// a_i <- (a_i * b_i - c_i) * zinv for plain Fr words: the pointwise step of a Groth16 witness
// map between the forward transforms on the coset g*H and the final inverse (z = g^N - 1 is
// the vanishing polynomial x^N - 1 evaluated anywhere on that coset). zinv2 holds zinv * R^2
// (Montgomery form of zinv times R), so three Montgomery products give the plain result:
//   u = a*b/R, w = c/R, (u - w) * zinv*R^2 / R = (a*b - c) * zinv.
// out may be a or c (each element is read before it is written, by the same thread).
__global__ void quotient_kernel(uint32_t* out, const uint32_t* a, const uint32_t* __restrict__ b, const uint32_t* c,
                                size_t n, Fr zinv2) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Fr v = quotient_element(load_fe<Fr>(a + 8 * i), load_fe<Fr>(b + 8 * i), load_fe<Fr>(c + 8 * i), zinv2);
  store_fe(out + 8 * i, v);
}

void quotient(uint32_t* out, const uint32_t* a, const uint32_t* b, const uint32_t* c, uint32_t log_n,
              const host::U256& zinv, cudaStream_t s) {
  const host::Field& f = host::fr();
  Fr z2;
  host::words32(host::to_mont(host::to_mont(zinv, f), f), z2.w);
  const size_t n = (size_t)1 << log_n;
  quotient_kernel<<<grid_for(n, 256), 256, 0, s>>>(out, a, b, c, n, z2);
  check_launch("quotient_kernel");
}

host::U256 coset_zinv(const uint32_t* g_plain, uint32_t log_n) {
  const host::Field& f = host::fr();
  const host::U256 g_raw = host::from_words32(g_plain);
  if (!(host::geq(f.p, g_raw) && !host::eq(f.p, g_raw))) fail(ZKG_EINVAL, "coset generator must be below r");
  const host::U256 g = host::to_mont(g_raw, f);
  const host::U256 gn = host::pow(g, host::U256{{(uint64_t)1 << log_n, 0, 0, 0}}, f);
  const host::U256 z = host::sub(gn, f.one, f);
  if (host::eq(z, host::U256{{0, 0, 0, 0}}))
    fail(ZKG_EINVAL, "g^N = 1: the coset is the subgroup itself and the vanishing polynomial is zero on it");
  return host::from_mont(host::inverse(z, f), f);
}

}  // namespace zkg

// ------------------------------------------------------------------ allocation-free entry point
//
// zkg_ntt_noalloc: the same transform for callers that cannot allocate device memory (code
// that runs under a memory budget owned by another allocator, inside a stream-ordered
// pipeline that forbids cudaMalloc, or in a process where only preallocated memory may be
// touched). Its scratch is a file-scope device array of fixed size instead of plan buffers.
namespace zkg {

constexpr uint32_t kNoAllocMaxLogN = ZKG_NTT_NOALLOC_MAX_LOG_N;
constexpr size_t kNoAllocPingPongWords = (size_t)8 << kNoAllocMaxLogN;         // 2 MiB
constexpr size_t kNoAllocTwiddleWords = (size_t)8 << (kNoAllocMaxLogN - 1);    // 1 MiB

// Every GPU that loads the library holds this array until the process exits. Nothing in it
// needs clearing: each call writes every word it reads (twiddles first, then pass 0 fills the
// ping-pong half before later passes read it).
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocPingPongWords + kNoAllocTwiddleWords];

// tw[j] = w^j (Montgomery form) by square-and-multiply over the bits of j.
__global__ void ntt_twiddles_pow(Fr w, uint32_t count, uint32_t* __restrict__ out) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= count) return;
  Fr acc = Fr::one(), base = w;
  for (uint32_t e = j; e; e >>= 1) {
    if (e & 1) acc = acc * base;
    base = base * base;
  }
  store_fe(out + 8 * (size_t)j, acc);
}

// Device address of g_noalloc_scratch per device, resolved with that device current (in host
// code the symbol names a host-side stand-in, not device memory). The cache is keyed on the
// device's current context as well: after cudaDeviceReset the device gets a new context, the
// old address is stale, and the next call resolves it again (and sets the kernels'
// shared-memory limit again, a per-context attribute).
static std::mutex g_noalloc_mutex;
struct NoAllocScratch {
  void* context;
  uint32_t* ptr;
};
static NoAllocScratch g_noalloc_cache[64];

using CtxGetCurrentFn = int (*)(void**);
static CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  if (!fn) fail(ZKG_ECUDA, "cuCtxGetCurrent is not available from the CUDA driver");
  return fn;
}

static uint32_t* noalloc_scratch(int device) {
  if (device < 0 || device >= 64) fail(ZKG_ENODEV, "device index out of range");
  void* context = nullptr;  // null before the runtime has made the device's context
  if (ctx_get_current()(&context) != 0) fail(ZKG_ECUDA, "cuCtxGetCurrent failed");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoAllocScratch& e = g_noalloc_cache[device];
  if (!e.ptr || !context || e.context != context) {
    void* p = nullptr;
    // The first runtime call that needs the device also makes its context current.
    check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(g_noalloc_scratch)");
    if (ctx_get_current()(&context) != 0 || !context) fail(ZKG_ECUDA, "no current CUDA context");
    set_pass_smem_limits();
    e.context = context;
    e.ptr = static_cast<uint32_t*>(p);
  }
  return e.ptr;
}

static void ntt_noalloc(uint32_t log_n, int inverse, uint32_t* data, cudaStream_t s) {
  if (log_n < 10 || log_n > kNoAllocMaxLogN)
    fail(ZKG_EINVAL, "log_n must be in 10..=" + std::to_string(kNoAllocMaxLogN) + " for zkg_ntt_noalloc, got " +
                         std::to_string(log_n));
  if (!data) fail(ZKG_EINVAL, "data is NULL");
  if ((reinterpret_cast<uintptr_t>(data) & 15) != 0) fail(ZKG_EINVAL, "data must be 16-byte aligned");
  int device = 0;
  check_cuda(cudaGetDevice(&device), "cudaGetDevice");
  uint32_t* scratch = noalloc_scratch(device);
  uint32_t* pingpong = scratch;
  uint32_t* tw = scratch + kNoAllocPingPongWords;

  const host::Field& f = host::fr();
  const size_t n = (size_t)1 << log_n;
  host::U256 w = host::root_of_unity(log_n);
  if (inverse) w = host::inverse(w, f);
  Fr wm, scale;
  host::words32(w, wm.w);
  host::words32(host::inverse(host::to_mont(host::U256{{(uint64_t)n, 0, 0, 0}}, f), f), scale.w);

  const uint32_t count = (uint32_t)(n / 2);
  ntt_twiddles_pow<<<grid_for(count, 256), 256, 0, s>>>(wm, count, tw);
  check_launch("ntt_twiddles_pow");

  // Same pass split and kernels as NttPlan (fixed arrays, no host allocation either).
  uint32_t passes[4], np = 0;
  if (log_n <= kTileLog) {
    passes[np++] = log_n;
  } else {
    uint32_t p = (log_n + kMaxStagesPerPass - 1) / kMaxStagesPerPass;
    for (uint32_t i = 0; i < p; i++) passes[np++] = log_n / p + (i < log_n % p ? 1u : 0u);
  }
  const uint32_t tl = log_n < kTileLog ? log_n : kTileLog;
  const unsigned tiles = 1u << (log_n - tl);
  const size_t smem = (size_t)32 << tl;
  uint32_t done = 0;
  for (uint32_t i = 0; i < np; i++) {
    const uint32_t st = passes[i];
    const uint32_t lm = log_n - done - st;
    const bool last = i + 1 == np;
    const uint32_t* src = i == 0 ? data : pingpong;
    uint32_t* dst = last ? data : pingpong;
    const int scale_flag = last && inverse;
    if (last)
      ntt_pass<true><<<tiles, kNttThreads, smem, s>>>(src, dst, tw, log_n, tl, lm, st, scale_flag, scale, nullptr,
                                                      nullptr, 0);
    else
      ntt_pass<false><<<tiles, kNttThreads, smem, s>>>(src, dst, tw, log_n, tl, lm, st, scale_flag, scale, nullptr,
                                                       nullptr, 0);
    check_launch("ntt_pass");
    done += st;
  }
}

}  // namespace zkg

extern "C" int zkg_ntt_noalloc(uint32_t log_n, int inverse, uint32_t* data, void* stream) {
  try {
    zkg::ntt_noalloc(log_n, inverse, data, static_cast<cudaStream_t>(stream));
    return ZKG_OK;
  } catch (const zkg::Error& e) {
    zkg::set_error(e.msg);
    return e.code;
  } catch (...) {
    zkg::set_error("unexpected internal error");
    return ZKG_ECUDA;
  }
}
