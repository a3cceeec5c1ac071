// Proving-request server (server.cu): resident proving keys, HBM-footprint admission and
// continuous batching of Groth16-shaped requests.
#pragma once
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "host_field.hpp"
#include "msm.hpp"
#include "ntt.hpp"
#include "runtime.hpp"

namespace zkg {

struct ServerKey {
  size_t n;
  const uint32_t* g1;  // n affine G1 points, Montgomery form
  const uint32_t* g2;  // n affine G2 points, Montgomery form
};

struct ServerRequest;

// Everything one request of size m = 2^log_m needs on the device, reused across requests.
struct ServerSlot {
  uint32_t log_m = 0;
  const ServerKey* key = nullptr;
  size_t bytes = 0;
  std::unique_ptr<MsmPlan> g1, g2;
  std::unique_ptr<NttPlan> ntt;
  std::unique_ptr<CosetShift> shift, unshift;
  DeviceArray sg1[3], sg2, poly[3], results;
  cudaStream_t stream = nullptr;
  cudaStream_t branch[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t graph_kernels = 0;
  bool busy = false;
  ServerRequest* req = nullptr;
  ~ServerSlot();
};

struct ServerRequest {
  uint64_t id = 0;
  zkg_proof_request desc;
  double t_submit = 0, t_start = 0, t_done = 0;
  int state = 0;  // 0 queued, 1 on the device, 2 done, 3 failed
  std::string error;
  ServerSlot* slot = nullptr;
  struct Server* server = nullptr;
};

struct Server {
  zkg_ctx* ctx;
  zkg_server_config cfg;
  host::U256 zinv;  // (g^N - 1)^-1 depends on N; computed per slot (see slot_zinv)
  std::vector<std::unique_ptr<ServerKey>> keys;
  std::vector<std::unique_ptr<ServerSlot>> slots;
  std::map<uint64_t, std::unique_ptr<ServerRequest>> requests;
  std::deque<ServerRequest*> queue;
  // admitted requests whose slot is being made, with the bytes reserved for it
  std::deque<std::pair<ServerRequest*, size_t>> builds;
  int building = 0;  // slots under construction (each holds a lane)
  // Per size: slots reserved by reserve(), slots under construction. A request whose size has
  // max(2, reserved) slots (built or being built), all busy, waits for one of them instead of
  // having another built: under load a build takes tens to hundreds of ms, longer than the wait.
  std::map<uint32_t, uint32_t> reserved, building_of;
  size_t bytes_used = 0, budget = 0;
  uint64_t next_id = 1;
  uint64_t slots_created = 0, slots_evicted = 0, completed = 0;
  double build_ms = 0;
  bool stopping = false;
  mutable std::mutex mu;
  std::condition_variable cv;  // queue, slot, build and completion changes
  std::thread dispatcher_thread, builder_thread;

  Server(zkg_ctx* ctx, const zkg_server_config& cfg);
  ~Server();
  int add_key(size_t n, const zkg_buf* g1, const zkg_buf* g2);
  uint64_t submit(const zkg_proof_request& r);
  int wait(uint64_t id, int timeout_ms, zkg_request_times* times);
  void stats(zkg_server_counters* s);
  void reserve(uint32_t log_m, uint32_t count);

 private:
  void dispatcher();
  void builder();
  std::unique_ptr<ServerSlot> make_slot(uint32_t log_m);
  size_t estimate_bytes(uint32_t log_m) const;
  const ServerKey* key_for(uint32_t log_m) const;
  void enqueue_work(ServerSlot* s, cudaStream_t main, cudaStream_t b0, cudaStream_t b1);
  void launch(ServerRequest* r, ServerSlot* s);
  static void CUDART_CB on_done(void* p);
};

}  // namespace zkg

struct zkg_server {
  zkg::Server server;
  zkg_server(zkg_ctx* ctx, const zkg_server_config& cfg) : server(ctx, cfg) {}
};
