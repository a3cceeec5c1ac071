// NTT plan (host side of Ntt, src/ntt.rs:14-119).
#pragma once
#include <vector>

#include "host_field.hpp"
#include "runtime.hpp"

namespace zkg {

struct NttPlan {
  zkg_ctx* ctx;
  uint32_t log_n;
  std::vector<uint32_t> passes;  // stages per pass
  uint32_t n_inv_words[8];       // 1/n in Montgomery form
  DeviceArray scratch, fwd_tw, inv_tw;
  StageTimer timer;  // one stage id per pass

  NttPlan(zkg_ctx* ctx, uint32_t log_n);
  // Queues one transform of data (2^log_n elements) on stream s.
  void enqueue(uint32_t* data, bool inverse, cudaStream_t s);
  void run(zkg_buf* data, bool inverse);

 private:
  void build_twiddles(const host::U256& root, DeviceArray& out);
};

}  // namespace zkg

struct zkg_ntt {
  zkg::NttPlan plan;
  zkg_ntt(zkg_ctx* ctx, uint32_t log_n) : plan(ctx, log_n) {}
};
