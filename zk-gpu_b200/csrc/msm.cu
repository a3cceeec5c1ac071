// MSM plan and driver: the host side of Msm (src/msm.rs:82-298), sm_100a kernels in
// msm_kernels.cuh.
//
// A plan owns every scratch buffer for a fixed (group, n, c, L); runs are queued on the
// context stream with no host synchronisation (data-dependent sizes such as the number of
// nonzero digits stay on the device: kernels read them and exit early), so a plan can be
// reused any number of times and captured in a CUDA graph.
#include <algorithm>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "host_field.hpp"
#include "msm.hpp"
#include "msm_f64.cuh"
#include "msm_kernels.cuh"

namespace zkg {

// Dynamic shared memory of msm_accumulate_f64: the G2 form keeps its accumulators there
// (4 coordinates x 10 doubles x 128 threads); G1 keeps them in registers.
template <class E>
static size_t f64_acc_smem(bool smem_acc = std::is_same<E, f64::Fq2D>::value) {
  return smem_acc ? (size_t)4 * f64::AccSmem<E>::N * 128 * sizeof(double) : 0;
}

// Allows the G2 form's dynamic shared memory beside its static staging buffers (72 KiB a block).
static void set_acc_smem_limits() {
  const int bytes = (int)f64_acc_smem<f64::Fq2D>();
  check_cuda(cudaFuncSetAttribute(msm_accumulate_f64<f64::Fq2D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes),
             "accumulation smem attribute");
  check_cuda(cudaFuncSetAttribute(msm_accumulate_f64<f64::Fq2D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  bytes),
             "accumulation smem attribute");
}

// The last reduction level's block holds one XYZZ point per thread in shared memory: 64 KiB for
// G2 (256 threads x 256 bytes), above the default limit.
static void set_scan_smem_limits() {
  const int bytes = (int)(kScanThreads * sizeof(Xyzz<Fq2CP>));
  check_cuda(cudaFuncSetAttribute(msm_reduce_scan<Fq2CP>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
             "reduction smem attribute");
}

uint32_t default_window(size_t n) {
  // clamp(log2(max(n,1)) - 5, 11, 16) (src/msm.rs:78-80)
  size_t v = n < 1 ? 1 : n;
  int lg = 63 - __builtin_clzll((unsigned long long)v);
  int c = lg - 5;
  if (c < 11) c = 11;
  if (c > 16) c = 16;
  return (uint32_t)c;
}

// Points accumulated per thread when the caller does not choose, by the number of (point,
// window) entries; measured on B200 (G1, uniform scalars, default windows with the GLV split,
// sweeping 8..256): 2^16 points (1.6M entries) best at 32 (1.26 ms against 1.34 at 16: fewer
// merge levels), 2^18 at 32, 2^20 at 64-128, 2^22 and 2^24 at 128; 2^14 at 8 (longer segments
// lengthen the accumulation chains, shorter ones add heads and merge levels).
static uint32_t auto_seg_len(size_t n, uint32_t windows) {
  const double entries = (double)n * windows;
  if (entries < (double)(1u << 19)) return 8;
  if (entries < (double)(1u << 23)) return 32;
  if (entries < (double)(1u << 26)) return 64;
  return 128;
}

MsmPlan::MsmPlan(zkg_ctx* c_, int group_, size_t n_, uint32_t c, uint32_t item_points)
    : ctx(c_), group(group_), n(n_), c(c) {
  if (n < 1) fail(ZKG_EINVAL, "an MSM needs at least one point");
  if (c < 9 || c > 20) fail(ZKG_EINVAL, "window size c must be in 9..=20, got " + std::to_string(c));
  if (group != ZKG_G1 && group != ZKG_G2) fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
  if (n >= (size_t)kNegBit) fail(ZKG_EINVAL, "an MSM holds fewer than 2^31 points");
  item_points_req = item_points;
  const size_t max_entries = (size_t)((255 + c - 1) / c) * n;

  use(ctx);
  if (group == ZKG_G2) {
    set_acc_smem_limits();
    set_scan_smem_limits();
  }
  glv = glv_default();
  // G1: FP64 limbs. With the GLV split one product per call at every size (measured: 2^16 1.27
  // against 1.28 ms for two per call, 2^20 5.48 / 5.58, 2^22 15.60 / 16.05); with the plain
  // windows two per call below 2^26 (window, point) entries, one above (3.5% faster at 2^20-2^21
  // points, equal at 2^22, 3.5% slower from 2^23).
  acc_variant = group == ZKG_G1 ? ((glv || (double)max_entries >= (double)(1u << 26)) ? 4 : 3) : 2;
  chunk = std::min(n, max_chunk());
  layout();
  result.alloc(xyzz_words(), "msm result");
  result_handle.ctx = ctx;
  result_handle.ptr = result.ptr;
  result_handle.words = xyzz_words();
  result_handle.owned = false;
  check_cuda(cudaMemsetAsync(result.ptr, 0, xyzz_words() * 4, ctx->stream), "msm result init");
}

size_t MsmPlan::max_chunk() const {
  // fewer than 2^32 - 1 (window, point) entries per pass; GLV: 2 chunk points below 2^31 too
  if (glv) return std::min<size_t>(0xfffffffeull / (2 * ((128 + c - 1) / c)), ((size_t)kNegBit >> 1) - 1);
  return 0xfffffffeull / ((255 + c - 1) / c);
}

void MsmPlan::set_chunk(size_t points) {
  if (fixed_base) fail(ZKG_EINVAL, "a fixed-base plan runs in one pass");
  use(ctx);
  chunk_req = points;
  const size_t want = std::min(n, std::min(points ? points : n, max_chunk()));
  if (want != chunk) {
    chunk = want;
    layout();
  }
}

void MsmPlan::layout() {
  const size_t np = glv ? 2 * chunk : chunk;  // points of the largest pass
  windows = glv ? (128 + c - 1) / c : (255 + c - 1) / c;
  half = 1u << (c - 1);
  slots = (size_t)windows * half;
  seg_len = item_points_req ? item_points_req : auto_seg_len(np, windows);
  const size_t xw = xyzz_words();
  const size_t max_entries = (size_t)windows * np;

  counts.alloc(slots, "msm counts");
  slot_start.alloc(slots + 1, "msm slot_start");
  cursor.alloc(slots, "msm cursor");
  scan_tiles_n = (uint32_t)((slots + kScanTile - 1) / kScanTile);
  if (scan_tiles_n > (uint32_t)kScanTile) fail(ZKG_EINVAL, "too many bucket slots");
  tile_sums.alloc(scan_tiles_n, "msm scan tiles");
  sorted.alloc(max_entries, "msm sorted");
  if (c <= 16) {
    ranks.alloc(max_entries, "msm ranks");
    digits.alloc((max_entries + 1) / 2, "msm ranked digits");  // 16 bits per entry
  }
  buckets.alloc(slots * xw, "msm buckets");

  heads_max = (max_entries + seg_len - 1) / seg_len;
  // Chains of the merge and running-sum levels. Merge: 4 heads per thread (twice the levels of
  // 16, a quarter of the chain; measured faster at every size, G1 2^24 1.43 -> 1.05 ms). Running
  // sums: chunks of 4 buckets below 2^23 entries, 8 above (measured: reduce + window sums at
  // G1 2^24 1.30 / 1.20 / 1.25 ms for chunks of 4 / 8 / 16, at 2^16 0.47 / 0.52 / 0.65 ms).
  merge_fan_in = 4;
  const uint32_t chunk_log = (double)max_entries < (double)(1u << 23) ? 2 : 3;
  size_t len = heads_max;
  merge_levels = 0;
  while (len > 1) {
    len = (len + merge_fan_in - 1) / merge_fan_in;
    merge_levels++;
  }
  size_t second = (heads_max + merge_fan_in - 1) / merge_fan_in;
  heads[0].alloc(heads_max * xw, "msm heads");
  head_keys[0].alloc(heads_max, "msm head keys");
  heads[1].alloc(std::max<size_t>(second, 1) * xw, "msm heads");
  head_keys[1].alloc(std::max<size_t>(second, 1), "msm head keys");

  // Running-sum levels: m_0 = B; m_{l+1} = ceil(m_l / C) - 1 while positive (C = 2^chunk_log).
  std::memset(&levels, 0, sizeof(levels));
  levels.chunk_log = chunk_log;
  const uint32_t bucket_chunk = 1u << chunk_log;
  uint32_t m = half;
  size_t tot_points = 0, run_points = 0;
  std::vector<uint32_t> ms;
  while (m > 0) {
    if (levels.count >= (uint32_t)kMaxReduceLevels) fail(ZKG_EINVAL, "too many reduction levels");
    if (m <= kScanLevelMax) {  // the last level: one block per window sums it whole (msm_reduce_scan)
      ms.push_back(m);
      levels.tot_len[levels.count] = 1;
      levels.tot_offset[levels.count] = (uint32_t)tot_points;
      tot_points += windows;
      levels.count++;
      break;
    }
    uint32_t chunks = (m + bucket_chunk - 1) / bucket_chunk;
    uint32_t blocks = (chunks + kReduceThreads - 1) / kReduceThreads;  // one tot point per block
    ms.push_back(m);
    levels.tot_len[levels.count] = blocks;
    levels.tot_offset[levels.count] = (uint32_t)tot_points;
    tot_points += (size_t)blocks * windows;
    m = chunks - 1;
    levels.count++;
    run_points = std::max<size_t>(run_points, (size_t)m * windows);
  }
  level_m = ms;
  tots.alloc(tot_points * xw, "msm tots");
  runs[0].alloc(std::max<size_t>(run_points, 1) * xw, "msm runs");
  runs[1].alloc(std::max<size_t>(run_points, 1) * xw, "msm runs");
  window_sums.alloc((size_t)windows * xw, "msm window sums");
  if (glv) glv_bases.alloc(chunk * affine_words(), "msm GLV bases (phi)");
  else glv_bases.release();
  if (passes() > 1) partial.alloc(xw, "msm pass result");
  else partial.release();
}

size_t MsmPlan::xyzz_words() const { return group == ZKG_G1 ? 32 : 64; }
size_t MsmPlan::affine_words() const { return group == ZKG_G1 ? 16 : 32; }

void MsmPlan::check_buffers(const zkg_buf* bases, const zkg_buf* scalars) const {
  // Msm::check_buffers (src/msm.rs:271-282): byte counts in the messages, like the reference.
  size_t sb = scalars->words * 4, need_s = n * 32;
  if (sb < need_s)
    fail(ZKG_ESIZE, "scalars buffer holds " + std::to_string(sb) + " bytes; " + std::to_string(n) +
                        " scalars need " + std::to_string(need_s));
  const size_t points = fixed_base ? (size_t)windows * n : n;  // a fixed-base table has a row per window
  size_t bb = bases->words * 4, need_b = points * affine_words() * 4;
  if (bb < need_b)
    fail(ZKG_ESIZE, "bases buffer holds " + std::to_string(bb) + " bytes; " + std::to_string(points) +
                        " points need " + std::to_string(need_b));
}

// GLV is the G1 default wherever it applies: measured faster than the plain windows at every
// default window on B200 (2^16: 1.35 against 1.69 ms; 2^18: 2.31 / 2.76; 2^20: 5.53 / 5.83;
// 2^22: 15.7 / 16.7; 2^24: 54.8 / 55.1), half the reduction and combination work for the same
// bucket additions.
bool MsmPlan::glv_default() const {
  return group == ZKG_G1 && c <= 16;
}

void MsmPlan::set_glv(bool enable) {
  if (enable == glv) return;
  if (enable) {
    if (group != ZKG_G1) fail(ZKG_EINVAL, "GLV splitting is for G1 (the endomorphism (x, y) -> (beta x, y))");
    if (c > 16) fail(ZKG_EINVAL, "GLV splitting needs a window size c <= 16, got " + std::to_string(c));
    if (fixed_base) fail(ZKG_EINVAL, "GLV splitting and fixed-base tables do not combine");
  }
  use(ctx);
  const bool old = glv;
  const size_t old_chunk = chunk;
  glv = enable;
  try {
    chunk = std::min(n, std::min(chunk_req ? chunk_req : n, max_chunk()));
    layout();
  } catch (...) {
    glv = old;
    chunk = old_chunk;
    layout();
    throw;
  }
}

void MsmPlan::set_fixed_base(bool enable) {
  if (enable && c > 16) fail(ZKG_EINVAL, "fixed-base tables need a window size c <= 16, got " + std::to_string(c));
  const size_t plain_windows = (255 + c - 1) / c;  // a table has a row per plain window
  if (enable && plain_windows * n >= (size_t)kNegBit)
    fail(ZKG_EINVAL, "a fixed-base table holds fewer than 2^31 points");
  if (enable && glv) set_glv(false);  // the table's rows are the plain windows
  if (enable && chunk != n) {  // one pass: the table's rows are n points apart
    chunk = n;
    layout();
  }
  fixed_base = enable;
}

void fixed_base_table(zkg_ctx* ctx, int group, const zkg_buf* bases, size_t n, uint32_t c, zkg_buf* out) {
  if (n < 1) fail(ZKG_EINVAL, "an MSM needs at least one point");
  if (c < 9 || c > 20) fail(ZKG_EINVAL, "window size c must be in 9..=20, got " + std::to_string(c));
  if (group != ZKG_G1 && group != ZKG_G2) fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
  const uint32_t windows = (255 + c - 1) / c;
  const size_t aw = group == ZKG_G1 ? 16 : 32;
  if (bases->words < n * aw) fail(ZKG_ESIZE, "bases buffer too small for n points");
  if (out->words < (size_t)windows * n * aw) fail(ZKG_ESIZE, "table buffer too small for windows * n points");
  use(ctx);
  if (group == ZKG_G1)
    msm_fixed_base_table<Fq><<<grid_for(n, 128), 128, 0, ctx->stream>>>(bases->ptr, n, c, windows, out->ptr);
  else
    msm_fixed_base_table<Fq2><<<grid_for(n, 128), 128, 0, ctx->stream>>>(bases->ptr, n, c, windows, out->ptr);
  check_launch("msm_fixed_base_table");
}

// The ranked sort's counting pass (msm_rank), plain or with the GLV split.
template <int AGG>
void MsmPlan::rank(const uint32_t* bases, const uint32_t* scalars, cudaStream_t s) {
  const unsigned b256 = 256;
  if (glv) {
    msm_glv_phi<<<grid_for(run_n, b256), b256, 0, s>>>(bases, run_n, glv_bases.ptr);
    check_launch("msm_glv_phi");
    msm_rank_glv<AGG><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, counts.ptr,
                                                              digits.as<uint16_t>(), ranks.ptr);
  } else {
    msm_rank<AGG><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, fixed_base, counts.ptr,
                                                          digits.as<uint16_t>(), ranks.ptr);
  }
}

template <class F>
void MsmPlan::stage(int which, const uint32_t* bases, const uint32_t* scalars, cudaStream_t s) {
  const unsigned b256 = 256;
  switch (which) {
    case kStageCount:
      check_cuda(cudaMemsetAsync(counts.ptr, 0, active_slots() * 4, s), "msm counts clear");
      if (ranked_sort()) {
        if (sort_agg == 0)
          rank<0>(bases, scalars, s);
        else if (sort_agg == 1)
          rank<1>(bases, scalars, s);
        else if (sort_agg == 2)
          rank<2>(bases, scalars, s);
        else
          rank<3>(bases, scalars, s);
        check_launch("msm_rank");
      } else if (sort_agg == 1)
        msm_count<1><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, counts.ptr);
      else if (sort_agg == 2)
        msm_count<2><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, counts.ptr);
      else if (sort_agg == 3)
        msm_count<3><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, counts.ptr);
      else
        msm_count<0><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, counts.ptr);
      check_launch("msm_count");
      break;
    case kStageScan:
    {
      const size_t ns = active_slots();
      const uint32_t tiles = (uint32_t)((ns + kScanTile - 1) / kScanTile);
      scan_tile_sums<<<tiles, kScanBlock, 0, s>>>(counts.ptr, ns, tile_sums.ptr);
      check_launch("scan_tile_sums");
      scan_tiles<<<1, kScanBlock, 0, s>>>(tile_sums.ptr, tiles, slot_start.ptr + ns);
      check_launch("scan_tiles");
      scan_apply<<<tiles, kScanBlock, 0, s>>>(counts.ptr, ns, tile_sums.ptr, slot_start.ptr, cursor.ptr,
                                                     0u);
      check_launch("scan_apply");
      break;
    }
    case kStageScatter:
      if (ranked_sort()) {
        const dim3 grid((unsigned)grid_for(points(), b256), windows);
        msm_place<<<grid, b256, 0, s>>>(digits.as<uint16_t>(), ranks.ptr, points(), half, fixed_base, glv ? 1 : 0,
                                        slot_start.ptr, sorted.ptr);
        check_launch("msm_place");
        break;
      }
      // every group merged: measured best or equal for the scatter on every distribution
      msm_scatter<0><<<grid_for(run_n, b256), b256, 0, s>>>(scalars, run_n, c, windows, cursor.ptr, sorted.ptr);
      check_launch("msm_scatter");
      break;
    case kStageAccumulate: {
      // GLV: points run_n..2 run_n - 1 are the phi(P_i) of glv_bases
      const uint32_t* bases2 = glv ? glv_bases.ptr : bases;
      const uint32_t split = glv ? (uint32_t)run_n : 0xffffffffu;
      if ((acc_variant == 5 || acc_variant == 6) && std::is_same<F, Fq>::value) {
        // G1 with the accumulator in shared memory, four blocks per SM
        const size_t acc_smem = f64_acc_smem<f64::FqD>(true);
        if (acc_variant == 5)
          msm_accumulate_f64<f64::FqD, false, true><<<grid_for(heads_max, 128), 128, acc_smem, s>>>(
              bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
        else
          msm_accumulate_f64<f64::FqD, true, true><<<grid_for(heads_max, 128), 128, acc_smem, s>>>(
              bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
      } else if (acc_variant >= 3) {
        using E = typename std::conditional<std::is_same<F, Fq>::value, f64::FqD, f64::Fq2D>::type;
        const size_t acc_smem = f64_acc_smem<E>();
        if (acc_variant == 3 || acc_variant == 6)
          msm_accumulate_f64<E, true><<<grid_for(heads_max, 128), 128, acc_smem, s>>>(
              bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
        else
          msm_accumulate_f64<E, false><<<grid_for(heads_max, 128), 128, acc_smem, s>>>(
              bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
      }
      else if (acc_variant == 1)
        msm_accumulate<typename CompactOf<F>::type><<<grid_for(heads_max, 128), 128, 0, s>>>(
            bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
      else if (acc_variant == 2)
        msm_accumulate<typename PairedOf<F>::type><<<grid_for(heads_max, 128), 128, 0, s>>>(
            bases, bases2, split, sorted.ptr, slot_start.ptr, (uint32_t)active_slots(), seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
      else
        msm_accumulate<F><<<grid_for(heads_max, 128), 128, 0, s>>>(bases, bases2, split, sorted.ptr, slot_start.ptr,
                                                                   (uint32_t)active_slots(),
                                                                   seg_len, buckets.ptr, heads[0].ptr, head_keys[0].ptr);
      check_launch("msm_accumulate");
      break;
    }
    case kStageCombine:
      // c (W - 1) dependent doublings: one warp, each level's independent products on separate
      // lanes. G1 inlines its products (measured 5-8% faster than one out-of-line product per
      // lane: 2^16 with GLV 0.287 -> 0.265 ms); G2 keeps the out-of-line Fq2 products.
      if constexpr (std::is_same<F, Fq>::value)
        msm_combine_lanes<Fq><<<1, 32, 0, s>>>(window_sums.ptr, active_windows(), glv ? 128u / windows : c,
                                               glv ? 128u % windows : 0u, combine_out);
      else
        msm_combine_lanes<typename CompactOf<F>::type><<<1, 32, 0, s>>>(window_sums.ptr, active_windows(),
                                                                         glv ? 128u / windows : c,
                                                                         glv ? 128u % windows : 0u, combine_out);
      check_launch("msm_combine_lanes");
      if (!first_pass) {  // a later pass: add its point into the result
        msm_add_partial<F><<<1, 32, 0, s>>>(result.ptr, partial.ptr);
        check_launch("msm_add_partial");
      }
      break;
    case kStageMerge:
    case kStageReduce:
    case kStageWindows:
      // Two products per out-of-line call in every form (measured faster than one per call for
      // both groups, although the paired Fq2 kernels spill, and than inlined products for G1:
      // 2^24 merge 1.10 -> 1.49 ms, reduce 0.66 -> 1.09 ms inlined).
      tail_stage<typename PairedOf<F>::type>(which, s);
      break;
  }
}

template <class FC>
void MsmPlan::tail_stage(int which, cudaStream_t s) {
  switch (which) {
    case kStageMerge: {
      size_t len = heads_max;  // the largest a level can be (the entry count is on the device)
      uint32_t l = 0;
      for (; l < merge_levels; l++) {
        size_t out_len = (len + merge_fan_in - 1) / merge_fan_in;
        if (out_len <= kMergeTailThreads) break;  // the rest in one block (msm_merge_tail)
        int src = l & 1, dst = src ^ 1;
        msm_merge<FC><<<grid_for(out_len, 128), 128, 0, s>>>(slot_start.ptr, (uint32_t)active_slots(), seg_len, merge_fan_in, l,
                                                            heads[src].ptr, head_keys[src].ptr, heads[dst].ptr,
                                                            head_keys[dst].ptr, buckets.ptr);
        check_launch("msm_merge");
        len = out_len;
      }
      if (l < merge_levels) {
        msm_merge_tail<FC><<<1, kMergeTailThreads, 0, s>>>(slot_start.ptr, (uint32_t)active_slots(), seg_len,
                                                         merge_fan_in, l, merge_levels - l, heads[0].ptr,
                                                         head_keys[0].ptr, heads[1].ptr, head_keys[1].ptr,
                                                         buckets.ptr);
        check_launch("msm_merge_tail");
      }
      break;
    }
    case kStageReduce: {
      const uint32_t* in = buckets.ptr;
      uint32_t in_stride = half;
      for (uint32_t l = 0; l < levels.count; l++) {
        uint32_t m = level_m[l];
        if (m <= kScanLevelMax) {  // the last level
          msm_reduce_scan<FC><<<active_windows(), kScanThreads, kScanThreads * sizeof(Xyzz<FC>), s>>>(
              in, in_stride, m, l == 0 ? slot_start.ptr : nullptr, tots.ptr + (size_t)levels.tot_offset[l] * xyzz_words(),
              levels.tot_len[l]);
          check_launch("msm_reduce_scan");
          break;
        }
        uint32_t chunks = (m + (1u << levels.chunk_log) - 1) >> levels.chunk_log;
        uint32_t* run_out = runs[l & 1].ptr;
        const dim3 grid(levels.tot_len[l], active_windows());
        msm_reduce_level<FC><<<grid, kReduceThreads, kReduceThreads * sizeof(Xyzz<FC>), s>>>(
            in, in_stride, m, levels.chunk_log, l == 0 ? slot_start.ptr : nullptr,
            tots.ptr + (size_t)levels.tot_offset[l] * xyzz_words(), levels.tot_len[l], run_out,
            chunks > 1 ? chunks - 1 : 1);
        check_launch("msm_reduce_level");
        in = run_out;
        in_stride = chunks > 1 ? chunks - 1 : 1;
      }
      break;
    }
    case kStageWindows: {
      msm_window_sums<FC><<<active_windows(), kWindowThreads, kWindowThreads * sizeof(Xyzz<FC>), s>>>(tots.ptr,
                                                                                                    levels,
                                                                                            window_sums.ptr);
      check_launch("msm_window_sums");
      break;
    }
    case kStageCombine:  // launched by stage() (msm_combine_lanes)
      break;
  }
}

const char* MsmPlan::stage_name(int which) {
  static const char* names[kStages] = {"count", "scan", "scatter", "accumulate", "merge", "reduce", "window sums", "combine"};
  return names[which];
}

// Selects pass `off` (its first point): run_n, where the combination writes, and the pass's
// slice of the bases (a fixed-base plan has one pass) and scalars.
void MsmPlan::begin_pass(size_t off, const uint32_t*& bases, const uint32_t*& scalars) {
  run_n = std::min(chunk, n - off);
  first_pass = off == 0;
  combine_out = first_pass ? result.ptr : partial.ptr;
  bases += off * affine_words();
  scalars += off * 8;
}

void MsmPlan::enqueue(const uint32_t* bases, const uint32_t* scalars, cudaStream_t s) {
  for (size_t off = 0; off < n; off += chunk) {
    const uint32_t *b = bases, *sc = scalars;
    begin_pass(off, b, sc);
    for (int st = 0; st < kStages; st++) {
      size_t ev = timer.enabled ? timer.begin(st, s) : 0;
      if (group == ZKG_G1) stage<Fq>(st, b, sc, s);
      else stage<Fq2>(st, b, sc, s);
      if (timer.enabled) timer.end(ev, s);
    }
  }
  if (timer.enabled) timer.runs++;
}

void MsmPlan::run(const zkg_buf* bases, const zkg_buf* scalars) {
  check_buffers(bases, scalars);
  use(ctx);
  enqueue(bases->ptr, scalars->ptr, ctx->stream);
}

std::vector<std::pair<std::string, double>> MsmPlan::profile(const zkg_buf* bases, const zkg_buf* scalars) {
  check_buffers(bases, scalars);
  use(ctx);
  std::vector<std::pair<std::string, double>> out;
  cudaEvent_t a, b;
  check_cuda(cudaEventCreate(&a), "event");
  check_cuda(cudaEventCreate(&b), "event");
  for (int st = 0; st < kStages; st++) out.emplace_back(stage_name(st), 0.0);
  for (size_t off = 0; off < n; off += chunk) {  // stage times summed over the passes
    const uint32_t *bp = bases->ptr, *sp = scalars->ptr;
    begin_pass(off, bp, sp);
    for (int st = 0; st < kStages; st++) {
      check_cuda(cudaEventRecord(a, ctx->stream), "event record");
      if (group == ZKG_G1) stage<Fq>(st, bp, sp, ctx->stream);
      else stage<Fq2>(st, bp, sp, ctx->stream);
      check_cuda(cudaEventRecord(b, ctx->stream), "event record");
      check_cuda(cudaEventSynchronize(b), "msm stage");
      float ms = 0;
      check_cuda(cudaEventElapsedTime(&ms, a, b), "event time");
      out[st].second += (double)ms;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return out;
}

// ------------------------------------------------------------------ GLV split check

// out[10 i ..]: |k1| (4 words), |k2| (4 words), sign of k1, sign of k2, by glv::split_half.
__global__ void glv_split_kernel(const uint32_t* __restrict__ scalars, size_t count, uint32_t* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  for (int h = 0; h < 2; h++) {
    uint32_t s[8];
    load_scalar(scalars, i, s);
    const bool neg = glv::split_half(s, h == 1);
    for (int k = 0; k < 4; k++) out[10 * i + 4 * h + k] = s[k];
    out[10 * i + 8 + h] = neg ? 1u : 0u;
  }
}

void glv_split(zkg_ctx* ctx, const uint32_t* scalars, size_t count, uint32_t* out) {
  use(ctx);
  DeviceArray in, res;
  in.alloc(count * 8, "GLV split input");
  res.alloc(count * 10, "GLV split output");
  check_cuda(cudaMemcpyAsync(in.ptr, scalars, count * 32, cudaMemcpyHostToDevice, ctx->stream), "copy");
  glv_split_kernel<<<grid_for(count, 128), 128, 0, ctx->stream>>>(in.ptr, count, res.ptr);
  check_launch("glv_split_kernel");
  check_cuda(cudaMemcpyAsync(out, res.ptr, count * 40, cudaMemcpyDeviceToHost, ctx->stream), "copy");
  check_cuda(cudaStreamSynchronize(ctx->stream), "GLV split");
}

// ------------------------------------------------------------------ base upload

// Rescales every coordinate in place on the device: v -> v * scale / 2^256.
static void rescale(zkg_ctx* ctx, zkg_buf* buf, const host::U256& scale_mont) {
  Fq s;
  host::words32(scale_mont, s.w);
  size_t coords = buf->words / 8;
  if (coords == 0) return;
  fq_rescale<<<grid_for(coords, 256), 256, 0, ctx->stream>>>(buf->ptr, coords, s);
  check_launch("fq_rescale");
}

void upload_bases(zkg_ctx* ctx, const uint32_t* xy, size_t words, bool mont256, zkg_buf* out) {
  (void)xy;
  (void)words;
  // Msm::upload_bases: scale = R^2 turns plain x into x*R (src/msm.rs:182-188).
  // Msm::upload_bases_montgomery_256: the input is x*2^256 = x*R already (src/msm.rs:190-197).
  if (!mont256) rescale(ctx, out, host::fq().r2);
}

}  // namespace zkg
