// Batched execution: many MSMs, NTTs and coset shifts of uneven sizes captured into one CUDA
// graph and replayed with a single launch (the plain form is one Msm::run / Ntt::forward per
// call, src/msm.rs:286, src/ntt.rs:52).
//
// Operations are recorded on "lanes". Operations in one lane run in order; different lanes
// are independent graph branches, so the device overlaps them (a lane per request lets the
// arithmetic of small requests fill the SMs that one request alone leaves idle). A plan owns
// its scratch, so one plan may appear in one lane only. MSM results are copied out of the
// plan's result buffer into a caller buffer inside the graph, so a plan can run several times
// in its lane.
#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "batch.hpp"
#include "msm.hpp"
#include "ntt.hpp"

namespace zkg {

void Batch::check_lane(const void* plan, int lane) {
  if (lane < 0 || lane >= (int)kMaxLanes) fail(ZKG_EINVAL, "lane must be in 0.." + std::to_string(kMaxLanes - 1));
  auto it = plan_lane.find(plan);
  if (it != plan_lane.end() && it->second != lane)
    fail(ZKG_EINVAL, "a plan can be used in one lane only (its scratch is not shared)");
  plan_lane[plan] = lane;
  lanes = std::max(lanes, lane + 1);
  dirty = true;
}

void Batch::add_msm(MsmPlan* plan, const zkg_buf* bases, const zkg_buf* scalars, zkg_buf* out, int lane) {
  plan->check_buffers(bases, scalars);
  bufs.push_back(bases);
  bufs.push_back(scalars);
  bufs.push_back(&plan->result_handle);  // the plan's own result, written by the batch too
  if (out) bufs.push_back(out);
  if (out && out->words < plan->xyzz_words()) fail(ZKG_ESIZE, "result buffer too small for one XYZZ point");
  check_lane(plan, lane);
  Op op;
  op.kind = Op::kMsm;
  op.lane = lane;
  op.msm = plan;
  op.a = bases->ptr;
  op.b = scalars->ptr;
  op.out = out ? out->ptr : nullptr;
  ops.push_back(op);
}

void Batch::add_ntt(NttPlan* plan, zkg_buf* data, bool inverse, int lane) {
  if (data->words < ((size_t)8 << plan->log_n)) fail(ZKG_ESIZE, "data buffer too small for the transform");
  bufs.push_back(data);
  check_lane(plan, lane);
  Op op;
  op.kind = inverse ? Op::kNttInverse : Op::kNttForward;
  op.lane = lane;
  op.ntt = plan;
  op.data = data->ptr;
  ops.push_back(op);
}

void Batch::add_coset(CosetShift* shift, zkg_buf* data, int lane) {
  if (data->words < ((size_t)8 << shift->log_n)) fail(ZKG_ESIZE, "data buffer too small for the coset shift");
  bufs.push_back(data);
  if (lane < 0 || lane >= (int)kMaxLanes) fail(ZKG_EINVAL, "lane out of range");
  lanes = std::max(lanes, lane + 1);
  dirty = true;
  Op op;
  op.kind = Op::kCoset;
  op.lane = lane;
  op.coset = shift;
  op.data = data->ptr;
  ops.push_back(op);
}

void Batch::enqueue_lane(int lane, cudaStream_t s) {
  for (const Op& op : ops) {
    if (op.lane != lane) continue;
    switch (op.kind) {
      case Op::kMsm: {
        bool timed = op.msm->timer.enabled;  // no stage events inside a batch
        op.msm->timer.enabled = false;
        op.msm->enqueue(op.a, op.b, s);
        op.msm->timer.enabled = timed;
        if (op.out)
          check_cuda(cudaMemcpyAsync(op.out, op.msm->result.ptr, op.msm->xyzz_words() * 4, cudaMemcpyDeviceToDevice, s),
                     "batch result copy");
        break;
      }
      case Op::kNttForward:
      case Op::kNttInverse: {
        bool timed = op.ntt->timer.enabled;
        op.ntt->timer.enabled = false;
        op.ntt->enqueue(op.data, op.kind == Op::kNttInverse, s);
        op.ntt->timer.enabled = timed;
        break;
      }
      case Op::kCoset:
        op.coset->enqueue(op.data, s);
        break;
    }
  }
}

void Batch::release_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
}

void Batch::ensure_streams() {
  while ((int)streams.size() < lanes) {
    cudaStream_t s;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch stream");
    streams.push_back(s);
    cudaEvent_t e;
    check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
    joins.push_back(e);
  }
  if (!fork) check_cuda(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "batch event");
}

// Captures all lanes into one graph: the context stream forks to one stream per lane and joins
// them back, so the graph's branches are the lanes.
void Batch::capture() {
  use(ctx);
  ensure_streams();
  release_graph();
  cudaStream_t origin = ctx->stream;
  check_cuda(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    check_cuda(cudaEventRecord(fork, origin), "fork");
    for (int l = 0; l < lanes; l++) {
      check_cuda(cudaStreamWaitEvent(streams[l], fork, 0), "fork wait");
      enqueue_lane(l, streams[l]);
      check_cuda(cudaEventRecord(joins[l], streams[l]), "join");
      check_cuda(cudaStreamWaitEvent(origin, joins[l], 0), "join wait");
    }
  } catch (...) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(origin, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    throw;
  }
  check_cuda(cudaStreamEndCapture(origin, &graph), "end capture");
  check_cuda(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
  graph_kernels = count_kernels();
  dirty = false;
}

void Batch::launch() {
  use(ctx);
  if (dirty || !exec) capture();
  for (const zkg_buf* b : bufs) wait_reads(b, ctx->stream);
  check_cuda(cudaGraphLaunch(exec, ctx->stream), "graph launch");
  for (const zkg_buf* b : bufs) mark_use(b, ctx->stream);
  // kernels inside the graph are this library's: count them like direct launches
  g_launches.fetch_add(graph_kernels, std::memory_order_relaxed);
}

// Runs the same operations without a graph: each lane on its own stream, forked from and
// joined back into the context stream (for comparison, and when capture is not wanted).
void Batch::run_streams() {
  use(ctx);
  ensure_streams();
  for (const zkg_buf* b : bufs) wait_reads(b, ctx->stream);
  check_cuda(cudaEventRecord(fork, ctx->stream), "fork");
  for (int l = 0; l < lanes; l++) {
    check_cuda(cudaStreamWaitEvent(streams[l], fork, 0), "fork wait");
    enqueue_lane(l, streams[l]);
    check_cuda(cudaEventRecord(joins[l], streams[l]), "join");
    check_cuda(cudaStreamWaitEvent(ctx->stream, joins[l], 0), "join wait");
  }
  for (const zkg_buf* b : bufs) mark_use(b, ctx->stream);
}

size_t Batch::count_kernels() const {
  if (!graph) return 0;
  size_t n = 0;
  if (cudaGraphGetNodes(graph, nullptr, &n) != cudaSuccess) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(graph, nodes.data(), &n) != cudaSuccess) return 0;
  size_t k = 0;
  for (auto node : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(node, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
  }
  return k;
}

Batch::~Batch() {
  release_graph();
  for (auto s : streams) cudaStreamDestroy(s);
  for (auto e : joins) cudaEventDestroy(e);
  if (fork) cudaEventDestroy(fork);
}

}  // namespace zkg
