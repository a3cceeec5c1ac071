// Constants and small structs shared by the MSM kernels (msm_kernels.cuh) and the host plan
// (msm.hpp).
#pragma once
#include <cstdint>

namespace zkg {

constexpr uint32_t kNegBit = 0x80000000u;
constexpr uint32_t kNoKey = 0xffffffffu;
// Heads summed per thread per merge level, and buckets per running-sum thread (2^chunk_log),
// chosen per plan: long chains suit many threads, short ones few (MsmPlan).
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;
constexpr int kWindowThreads = 128;
constexpr int kReduceThreads = 128;  // one running-sum block covers this many chunks of one window
constexpr int kMaxReduceLevels = 16;
// The last running-sum level takes at most this many values per window and is summed by one
// block (msm_reduce_scan) instead of further levels.
constexpr uint32_t kScanLevelMax = 1024;
constexpr int kScanThreads = 256;

struct ReduceLevels {
  uint32_t count;                         // levels
  uint32_t chunk_log;                     // buckets per running-sum thread = 2^chunk_log
  uint32_t tot_len[kMaxReduceLevels];     // tot values per window at each level
  uint32_t tot_offset[kMaxReduceLevels];  // start (in points) of level l's tot array; window stride = tot_len
};

}  // namespace zkg
