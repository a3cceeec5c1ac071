// Autotuner: measures candidate launch parameters on the device and returns the
// fastest. The reference fixes its parameters (Msm::default_window, src/msm.rs:78-80; item size
// mean_bucket/4, :99-100; TILE_LOG = 9 for the NTT, src/ntt.rs:9) and sweeps windows by hand
// (examples/g2_window.rs:50-69); default_window stays the plain form beside the tuned one.
//
// MSM candidates: window c in [default - 2, default + 2] within 9..=20, points per accumulation
// thread in {16, 32, 64, 128, 256}, the accumulation kernel forms, and for G1 (c <= 16) the GLV
// split on and off. NTT candidates: the most
// stages per shared-memory pass (passes = ceil(log_n / max_stages)). Each candidate runs once to
// warm up, then `reps` times between CUDA events; the best mean wins.
#include <algorithm>
#include <memory>
#include <vector>

#include "msm.hpp"
#include "ntt.hpp"
#include "tuning.hpp"

namespace zkg {

static double time_ms(cudaStream_t s, int reps, const std::function<void()>& fn) {
  cudaEvent_t a, b;
  check_cuda(cudaEventCreate(&a), "event");
  check_cuda(cudaEventCreate(&b), "event");
  fn();
  check_cuda(cudaEventRecord(a, s), "event");
  for (int i = 0; i < reps; i++) fn();
  check_cuda(cudaEventRecord(b, s), "event");
  check_cuda(cudaEventSynchronize(b), "tuning run");
  float ms = 0;
  check_cuda(cudaEventElapsedTime(&ms, a, b), "event");
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

std::vector<zkg_msm_tuning> tune_msm(zkg_ctx* ctx, int group, size_t n, const zkg_buf* bases,
                                     const zkg_buf* scalars, int reps) {
  use(ctx);
  const int c0 = (int)default_window(n);
  std::vector<zkg_msm_tuning> out;
  for (int c = std::max(9, c0 - 2); c <= std::min(20, c0 + 2); c++) {
    // G1 with c <= 16 also with the GLV split (2n points, ceil(128 / c) windows)
    for (int glv = 0; glv <= (group == ZKG_G1 && c <= 16 ? 1 : 0); glv++) {
      const uint32_t windows = glv ? (128 + c - 1) / c : (255 + c - 1) / c;
      const double entries = (double)n * (glv ? 2 : 1) * windows;
      for (uint32_t L : {16u, 32u, 64u, 128u, 256u}) {
        // keep at least a few waves of threads on 148 SMs
        if (entries / L < 148.0 * 256 && L > 16) continue;
        std::unique_ptr<MsmPlan> plan;
        try {
          plan.reset(new MsmPlan(ctx, group, n, (uint32_t)c, L));
          plan->set_glv(glv != 0);
        } catch (const Error& e) {
          if (e.code == ZKG_ENOMEM) {
            cudaGetLastError();
            continue;
          }
          throw;
        }
        plan->check_buffers(bases, scalars);
        // forms that can win: out-of-line integer products (1, 2) and, for G1, double-precision
        // limbs (3, 4); fully inlined products (0) lose to both everywhere measured
        const std::vector<int> variants = group == ZKG_G1 ? std::vector<int>{1, 2, 3, 4} : std::vector<int>{1, 2};
        for (int v : variants) {
          plan->acc_variant = v;
          double ms = time_ms(ctx->stream, reps, [&] { plan->enqueue(bases->ptr, scalars->ptr, ctx->stream); });
          out.push_back(zkg_msm_tuning{(uint32_t)c, L, v, glv, ms});
        }
      }
    }
  }
  std::sort(out.begin(), out.end(), [](const zkg_msm_tuning& a, const zkg_msm_tuning& b) { return a.ms < b.ms; });
  return out;
}

std::vector<NttChoice> tune_ntt(zkg_ctx* ctx, uint32_t log_n, zkg_buf* data, int reps) {
  use(ctx);
  std::unique_ptr<NttPlan> plan(new NttPlan(ctx, log_n));
  if (data->words < ((size_t)8 << log_n)) fail(ZKG_ESIZE, "data buffer too small for the transform");
  std::vector<NttChoice> out;
  for (int v = 0; v <= 4; v++) {
    plan->set_variant(v);
    const uint32_t tlog = plan->tile_log();
    for (uint32_t s = 6; s <= tlog; s++) {
      if (!plan->set_max_stages(s)) continue;
      if (plan->passes.size() == 1 && s != tlog) continue;  // one tile: every split is the same
      double ms = time_ms(ctx->stream, reps, [&] {
        plan->enqueue(data->ptr, false, ctx->stream);
        plan->enqueue(data->ptr, true, ctx->stream);
      });
      out.push_back(NttChoice{v, s, ms / 2});
    }
  }
  std::sort(out.begin(), out.end(), [](const NttChoice& a, const NttChoice& b) { return a.ms < b.ms; });
  return out;
}

}  // namespace zkg
