// Batched execution (batch.cu).
#pragma once
#include <map>
#include <vector>

#include "runtime.hpp"

namespace zkg {

struct MsmPlan;
struct NttPlan;
struct CosetShift;

struct Batch {
  static constexpr unsigned kMaxLanes = 64;
  struct Op {
    enum Kind { kMsm, kNttForward, kNttInverse, kCoset } kind;
    int lane = 0;
    MsmPlan* msm = nullptr;
    NttPlan* ntt = nullptr;
    CosetShift* coset = nullptr;
    const uint32_t* a = nullptr;  // MSM bases
    const uint32_t* b = nullptr;  // MSM scalars
    uint32_t* out = nullptr;      // MSM result copy target (may be null)
    uint32_t* data = nullptr;     // NTT / coset data
  };

  zkg_ctx* ctx;
  std::vector<Op> ops;
  std::vector<const zkg_buf*> bufs;  // every buffer the operations use (marked at each launch)
  std::map<const void*, int> plan_lane;
  int lanes = 0;
  bool dirty = true;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t graph_kernels = 0;

  explicit Batch(zkg_ctx* c) : ctx(c) {}
  ~Batch();
  void add_msm(MsmPlan* plan, const zkg_buf* bases, const zkg_buf* scalars, zkg_buf* out, int lane);
  void add_ntt(NttPlan* plan, zkg_buf* data, bool inverse, int lane);
  void add_coset(CosetShift* shift, zkg_buf* data, int lane);
  void capture();
  void launch();
  void run_streams();
  size_t kernels_per_launch() const { return graph_kernels; }

 private:
  void check_lane(const void* plan, int lane);
  void enqueue_lane(int lane, cudaStream_t s);
  void ensure_streams();
  void release_graph();
  size_t count_kernels() const;
};

}  // namespace zkg

struct zkg_batch {
  zkg::Batch batch;
  explicit zkg_batch(zkg_ctx* ctx) : batch(ctx) {}
};
