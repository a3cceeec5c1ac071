// MSM plan (host side of Msm, src/msm.rs:25-298).
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "msm_common.hpp"
#include "runtime.hpp"

namespace zkg {

uint32_t default_window(size_t n);
void upload_bases(zkg_ctx* ctx, const uint32_t* xy, size_t words, bool mont256, zkg_buf* out);
// out (windows * n points) <- the fixed-base table of n resident bases for window size c: row w
// holds 2^(c w) P_i (windows = ceil(255 / c)); queued on the context stream.
void fixed_base_table(zkg_ctx* ctx, int group, const zkg_buf* bases, size_t n, uint32_t c, zkg_buf* out);
// The device's GLV split of `count` host scalars (8 words each): per scalar |k1| and |k2| (4
// words each) and their signs (1 word each), to host memory.
void glv_split(zkg_ctx* ctx, const uint32_t* scalars, size_t count, uint32_t* out);

struct MsmPlan {
  enum Stage {
    kStageCount,
    kStageScan,
    kStageScatter,
    kStageAccumulate,
    kStageMerge,
    kStageReduce,
    kStageWindows,
    kStageCombine,
    kStages
  };

  zkg_ctx* ctx;
  int group;
  size_t n;
  uint32_t c, windows = 0, half = 0, seg_len = 0;
  // Accumulation kernel form: 0 = field products inlined, 1 = through one out-of-line product
  // (smaller code: the inlined mixed addition is thousands of instructions and its warps stall
  // on instruction fetch; measured 17% faster at 2^24), 2 = out of line, independent products
  // two per call, 3 / 4 = bucket arithmetic in double-precision limbs (msm_f64.cuh), two
  // products per call / one. Every form fetches the next base into shared memory with
  // cp.async. Defaults (measured on B200): G1 with the GLV split 4 at every size (2^20: 3.84
  // against 3.95 ms for 3); G1 with the plain windows 3 below 2^26 (window, point) entries and 4
  // above (2^24: 48.1 ms against 50.1 for 3 and 59.7 for 2; 2^20: 3.98 against 4.11 for 4), G2 2
  // (47.4 ms at 2^22 against 48.1 for 1 and 55.9 / 63.0 for the limb forms 4 / 3). Tunable.
  int acc_variant = 4;
  // Warp aggregation of the counting pass's atomics (slot_peers in msm_kernels.cuh): 0 = every
  // group of equal slots, 1 = the first lane's group, 2 = none, 3 = the group of the first equal
  // neighbour pair. The scatter pass always merges every group.
  int sort_agg = 3;
  // Counting sort: 0 = scalar-major scatter through atomic cursors, 1 = ranked (the counting
  // pass records each digit's rank in its slot, the placing pass runs window by window;
  // msm_rank / msm_place). 1 is the default where it applies (c <= 16).
  int sort_form = 1;
  bool ranked_sort() const { return fixed_base || glv || (sort_form == 1 && c <= 16); }
  // Fixed-base mode: `bases` of run() is a table from fixed_base_table() (windows * n points,
  // row w = 2^(c w) P_i), every window's digits share one set of 2^(c-1) buckets, and the
  // result is that set's running sum: no per-window reductions and no combination doublings.
  // Needs c <= 16 (the ranked sort).
  bool fixed_base = false;
  // GLV mode (G1, c <= 16): every scalar splits as k1 + k2 lambda with 127-bit halves, and the
  // MSM runs over the 2n points P_i, phi(P_i) (phi(P_i) in glv_bases, made from `bases` on every
  // run; each half-scalar's sign in its digits) with
  // W = ceil(128 / c) windows of floor(128 / W) or floor(128 / W) + 1 bits (glv_window_width):
  // about the same number of bucket additions, half the windows, so half the reductions and half
  // the combination doublings.
  // On by default where it applies (glv_default); zkg_msm_set_glv switches it; fixed-base mode
  // switches it off.
  bool glv = false;
  bool glv_default() const;
  // Points per pass. Entry positions and point indices are 32-bit, so one pass holds fewer than
  // 2^32 (window, point) entries; a run over more points goes in passes of `chunk` points whose
  // results are added (the reference's limit, n < 2^31, is kept). The plan's scratch is sized
  // for one pass, so a smaller chunk (zkg_msm_set_chunk) also bounds its device memory.
  size_t chunk = 0, run_n = 0;  // run_n: the points of the pass being queued
  size_t chunk_req = 0;         // 0: the largest pass the mode allows
  size_t max_chunk() const;
  void set_chunk(size_t points);
  size_t passes() const { return (n + chunk - 1) / chunk; }
  size_t points() const { return glv ? 2 * run_n : run_n; }
  size_t active_slots() const { return fixed_base ? half : slots; }
  uint32_t active_windows() const { return fixed_base ? 1u : windows; }
  size_t slots = 0, heads_max = 0;
  uint32_t merge_levels = 0, merge_fan_in = 16, scan_tiles_n = 0;
  ReduceLevels levels;
  std::vector<uint32_t> level_m;

  DeviceArray counts, slot_start, cursor, tile_sums, sorted, buckets;
  DeviceArray ranks, digits;  // the ranked sort's rank (32 bits) and digit (16 bits) per (window, point), window-major
  DeviceArray glv_bases;      // GLV mode: phi(P_0)..phi(P_{n-1})
  DeviceArray heads[2], head_keys[2];
  DeviceArray tots, runs[2], window_sums, result, partial;  // partial: a later pass's result
  zkg_buf result_handle;
  StageTimer timer;

  MsmPlan(zkg_ctx* ctx, int group, size_t n, uint32_t c, uint32_t item_points);
  ~MsmPlan() {
    if (result_handle.last_use) cudaEventDestroy(result_handle.last_use);
    if (result_handle.pending_read) cudaEventDestroy(result_handle.pending_read);
  }
  MsmPlan(const MsmPlan&) = delete;
  MsmPlan& operator=(const MsmPlan&) = delete;
  size_t xyzz_words() const;
  size_t affine_words() const;
  void check_buffers(const zkg_buf* bases, const zkg_buf* scalars) const;
  void set_fixed_base(bool enable);
  void set_glv(bool enable);
  // Queues every stage on stream s (no host synchronisation).
  void enqueue(const uint32_t* bases, const uint32_t* scalars, cudaStream_t s);
  void run(const zkg_buf* bases, const zkg_buf* scalars);
  std::vector<std::pair<std::string, double>> profile(const zkg_buf* bases, const zkg_buf* scalars);
  static const char* stage_name(int which);

 private:
  template <class F>
  void stage(int which, const uint32_t* bases, const uint32_t* scalars, cudaStream_t s);
  template <class FC>
  void tail_stage(int which, cudaStream_t s);
  // Windows, slots, segments, merge and reduction levels and their scratch, for the current
  // mode (points() and the scalar width); the result buffer is kept.
  void layout();
  uint32_t* combine_out = nullptr;  // where the combination of the pass being queued goes
  bool first_pass = true;
  void begin_pass(size_t off, const uint32_t*& bases, const uint32_t*& scalars);
  template <int AGG>
  void rank(const uint32_t* bases, const uint32_t* scalars, cudaStream_t s);
  uint32_t item_points_req = 0;
};

}  // namespace zkg

struct zkg_msm {
  zkg::MsmPlan plan;
  template <class... A>
  explicit zkg_msm(A&&... a) : plan(std::forward<A>(a)...) {}
};
