// Autotuner (tuning.cu).
#pragma once
#include <functional>
#include <utility>
#include <vector>

#include "runtime.hpp"

namespace zkg {

std::vector<zkg_msm_tuning> tune_msm(zkg_ctx* ctx, int group, size_t n, const zkg_buf* bases, const zkg_buf* scalars,
                                     int reps);
struct NttChoice {
  int variant;
  uint32_t max_stages;
  double ms;  // per transform
};
std::vector<NttChoice> tune_ntt(zkg_ctx* ctx, uint32_t log_n, zkg_buf* data, int reps);

}  // namespace zkg
