// Proving-request server: the serving form of the hot path (the reference has no server, its
// callers issue one Msm::run / Ntt::forward at a time, src/msm.rs:286, src/ntt.rs:43-50).
//
// A request is Groth16-shaped: three G1 MSMs (sizes m, m, m - 1024) and one G2 MSM (size m) over
// the smallest resident proving key with at least m points, and a witness-map chain of seven
// Fr NTTs of size N = 2m on three evaluation vectors a, b, c:
//   for p in (a, b, c): p <- forward(coset_shift_g(inverse(p)))         (6 NTTs)
//   h <- (a * b - c) / (g^N - 1)   pointwise on the coset
//   h <- coset_shift_{1/g}(inverse(h))                                   (7th NTT)
// Outputs: the four MSM results (XYZZ words) and the N coefficients of h.
//
// Slots: the plans and device buffers one request of size class log_m needs, created on demand
// and reused. Admission: a request leaves the FIFO queue when a free slot of its size exists,
// or when a new one fits the HBM budget (idle slots of other sizes are evicted to make room)
// and fewer than `lanes` requests are on the device. Continuous batching: every slot has its
// own stream, so requests admitted while others run overlap on the device; in served mode a
// request's compute is one CUDA graph, captured when its slot is made, with three parallel
// branches (G1 MSMs, G2 MSM, NTT chain). Plain mode is the one-call-at-a-time path: one
// request on the device at a time, every operation launched directly, no branches.
//
// The dispatcher never calls CUDA while holding the mutex: completion callbacks
// (cudaLaunchHostFunc) take the mutex, and some CUDA calls wait for pending callbacks.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>

#include "server.hpp"

namespace zkg {

static double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Text of the exception being handled (inside a catch block): a failed request records it
// instead of letting the exception leave a server thread, which would end the process.
static std::string current_error_text() {
  try {
    throw;
  } catch (const Error& e) {
    return e.msg;
  } catch (const std::exception& e) {
    return std::string("internal error: ") + e.what();
  } catch (...) {
    return "unexpected internal error";
  }
}

ServerSlot::~ServerSlot() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (auto s : branch)
    if (s) cudaStreamDestroy(s);
  if (stream) cudaStreamDestroy(stream);
  if (fork) cudaEventDestroy(fork);
  for (auto e : join)
    if (e) cudaEventDestroy(e);
}

Server::Server(zkg_ctx* c, const zkg_server_config& config) : ctx(c), cfg(config) {
  if (cfg.lanes < 1 || cfg.lanes > 64) fail(ZKG_EINVAL, "lanes must be in 1..=64");
  if (cfg.plain) cfg.lanes = 1;
  host::U256 g = host::from_words32(cfg.coset_g);
  if (host::is_zero(g) || host::geq(g, host::fr().p)) fail(ZKG_EINVAL, "coset generator must be in 1..r-1");
  use(ctx);
  budget = cfg.hbm_budget_bytes;
  if (budget == 0) {
    size_t free_b = 0, total = 0;
    check_cuda(cudaMemGetInfo(&free_b, &total), "cudaMemGetInfo");
    budget = free_b / 10 * 8;
  }
  dispatcher_thread = std::thread([this] { dispatcher(); });
  builder_thread = std::thread([this] { builder(); });
}

Server::~Server() {
  {
    std::lock_guard<std::mutex> lock(mu);
    stopping = true;
  }
  cv.notify_all();
  if (dispatcher_thread.joinable()) dispatcher_thread.join();
  cv.notify_all();
  if (builder_thread.joinable()) builder_thread.join();
  cudaSetDevice(ctx->device);
  for (auto& s : slots)
    if (s->stream) cudaStreamSynchronize(s->stream);
}

int Server::add_key(size_t n, const zkg_buf* g1, const zkg_buf* g2) {
  if (n == 0) fail(ZKG_EINVAL, "a proving key needs at least one point");
  if (g1->words < 16 * n) fail(ZKG_ESIZE, "G1 bases buffer too small for the key");
  if (g2->words < 32 * n) fail(ZKG_ESIZE, "G2 bases buffer too small for the key");
  std::lock_guard<std::mutex> lock(mu);
  keys.push_back(std::unique_ptr<ServerKey>(new ServerKey{n, g1->ptr, g2->ptr}));
  return (int)keys.size() - 1;
}

// Takes mu: add_key may grow the key list from another thread at the same time. The keys
// themselves live behind unique_ptr, so the pointer returned stays valid after the lock ends.
const ServerKey* Server::key_for(uint32_t log_m) const {
  std::lock_guard<std::mutex> lock(mu);
  const ServerKey* best = nullptr;
  const size_t m = (size_t)1 << log_m;
  for (auto& k : keys)
    if (k->n >= m && (!best || k->n < best->n)) best = k.get();
  return best;
}

// Device bytes of a slot, from the same formulas the plans allocate with.
size_t Server::estimate_bytes(uint32_t log_m) const {
  const size_t m = (size_t)1 << log_m, N = 2 * m;
  auto msm = [&](size_t xw) {
    const uint32_t c = default_window(m), W = (255 + c - 1) / c;
    const bool glv = xw == 32 && c <= 16;  // G1 plans split with GLV by default
    const uint32_t Wg = (128 + c - 1) / c;
    const size_t B = (size_t)1 << (c - 1), S = (size_t)W * B;
    // (point, window) entries: the GLV plan has Wg windows over 2m points
    const size_t entries = std::max((size_t)W * m, glv ? (size_t)Wg * 2 * m : 0), L = 8;  // worst-case segment
    const size_t heads = entries / L + 1;
    // counts, slot starts, cursors; sorted entries, ranks and digits; buckets; heads; running
    // sums; the GLV bases (phi of the m points)
    return 4 * (3 * S + entries * 5 / 2 + S * xw + (heads + heads / 16 + 2) * (xw + 1) + 8 * W * B / 16 * xw / 8 +
                (glv ? m * 16 : 0) + 4096);
  };
  // scratch, twiddle words (both directions), staged twiddle tables (both directions: 40 bytes
  // per element for the first pass, at most as much again for the later passes' small tables
  // at these sizes) or the twiddle limbs of form 1 (20 bytes per element per direction)
  const size_t ntt = 32 * N + 2 * 16 * N + 2 * 48 * N;
  const size_t bufs = 3 * 32 * m + 32 * m + 3 * 32 * N + 4096;
  return msm(32) + msm(64) + ntt + bufs;
}


std::unique_ptr<ServerSlot> Server::make_slot(uint32_t log_m) {
  use(ctx);
  std::unique_ptr<ServerSlot> s(new ServerSlot);
  s->log_m = log_m;
  s->key = key_for(log_m);
  if (!s->key) fail(ZKG_EINVAL, "no resident proving key has 2^" + std::to_string(log_m) + " points");
  const size_t m = (size_t)1 << log_m, N = 2 * m;
  size_t free0 = 0, free1 = 0, total = 0;
  check_cuda(cudaMemGetInfo(&free0, &total), "cudaMemGetInfo");
  s->g1.reset(new MsmPlan(ctx, ZKG_G1, m, default_window(m), 0));
  s->g2.reset(new MsmPlan(ctx, ZKG_G2, m, default_window(m), 0));
  s->ntt.reset(new NttPlan(ctx, log_m + 1));
  s->shift.reset(new CosetShift(ctx, log_m + 1, cfg.coset_g));
  // 1/g as plain words for the unshift
  {
    const host::Field& f = host::fr();
    host::U256 gi = host::from_mont(host::inverse(host::to_mont(host::from_words32(cfg.coset_g), f), f), f);
    uint32_t w[8];
    host::words32(gi, w);
    s->unshift.reset(new CosetShift(ctx, log_m + 1, w));
  }
  s->ntt->prepare_shift(*s->shift);  // tables of the fused shifts, made before graph capture
  s->ntt->prepare_shift(*s->unshift);
  for (auto& b : s->sg1) b.alloc(8 * m, "server scalars");
  s->sg2.alloc(8 * m, "server scalars");
  for (auto& p : s->poly) p.alloc(8 * N, "server polynomials");
  s->results.alloc(3 * 32 + 64, "server results");
  check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "slot stream");
  for (auto& b : s->branch) check_cuda(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking), "slot stream");
  check_cuda(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming), "slot event");
  for (auto& e : s->join) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "slot event");
  if (!cfg.plain) {
    // One graph for the request's compute: three branches forked from the slot stream.
    check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "slot capture");
    try {
      enqueue_work(s.get(), s->stream, s->branch[0], s->branch[1]);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s->stream, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    check_cuda(cudaStreamEndCapture(s->stream, &s->graph), "slot capture");
    check_cuda(cudaGraphInstantiate(&s->exec, s->graph, 0), "slot graph instantiate");
    size_t nodes = 0;
    if (cudaGraphGetNodes(s->graph, nullptr, &nodes) == cudaSuccess) {
      std::vector<cudaGraphNode_t> v(nodes);
      cudaGraphGetNodes(s->graph, v.data(), &nodes);
      for (auto nd : v) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) s->graph_kernels++;
      }
    }
  }
  check_cuda(cudaStreamSynchronize(s->stream), "slot set-up");
  check_cuda(cudaMemGetInfo(&free1, &total), "cudaMemGetInfo");
  s->bytes = free0 > free1 ? free0 - free1 : estimate_bytes(log_m);
  return s;
}

void Server::enqueue_work(ServerSlot* s, cudaStream_t main, cudaStream_t b0, cudaStream_t b1) {
  const bool fork = b0 != main;
  if (fork) {
    check_cuda(cudaEventRecord(s->fork, main), "fork");
    check_cuda(cudaStreamWaitEvent(b0, s->fork, 0), "fork");
    check_cuda(cudaStreamWaitEvent(b1, s->fork, 0), "fork");
  }
  // G1: three MSMs on one plan, results copied out in turn
  for (int j = 0; j < 3; j++) {
    s->g1->enqueue(s->key->g1, s->sg1[j].ptr, main);
    check_cuda(cudaMemcpyAsync(s->results.ptr + 32 * j, s->g1->result.ptr, 32 * 4, cudaMemcpyDeviceToDevice, main),
               "result copy");
  }
  // G2
  s->g2->enqueue(s->key->g2, s->sg2.ptr, b0);
  check_cuda(cudaMemcpyAsync(s->results.ptr + 96, s->g2->result.ptr, 64 * 4, cudaMemcpyDeviceToDevice, b0),
             "result copy");
  // witness-map chain
  const uint32_t log_n = s->log_m + 1;
  for (int j = 0; j < 3; j++)
    s->ntt->enqueue(s->poly[j].ptr, true, b1, s->shift.get());  // inverse, then shift by g in its last pass
  s->ntt->enqueue(s->poly[0].ptr, false, b1);
  s->ntt->enqueue(s->poly[1].ptr, false, b1);
  // c's forward transform ends with h = (a b - c) / (g^N - 1), written over c
  const Quotient q{s->poly[0].ptr, s->poly[1].ptr, coset_zinv(cfg.coset_g, log_n)};
  s->ntt->enqueue(s->poly[2].ptr, false, b1, nullptr, &q);
  s->ntt->enqueue(s->poly[2].ptr, true, b1, s->unshift.get());
  if (fork) {
    check_cuda(cudaEventRecord(s->join[0], b0), "join");
    check_cuda(cudaEventRecord(s->join[1], b1), "join");
    check_cuda(cudaStreamWaitEvent(main, s->join[0], 0), "join");
    check_cuda(cudaStreamWaitEvent(main, s->join[1], 0), "join");
  }
}

void CUDART_CB Server::on_done(void* p) {
  // Runs on a CUDA callback thread: no CUDA calls here.
  ServerRequest* r = static_cast<ServerRequest*>(p);
  Server* sv = r->server;
  {
    std::lock_guard<std::mutex> lock(sv->mu);
    r->t_done = now_ms();
    r->state = 2;
    if (r->slot) {
      r->slot->busy = false;
      r->slot->req = nullptr;
    }
    sv->completed++;
  }
  sv->cv.notify_all();
}

void Server::launch(ServerRequest* r, ServerSlot* s) {
  use(ctx);
  const zkg_proof_request& d = r->desc;
  const size_t m = (size_t)1 << s->log_m, N = 2 * m;
  cudaStream_t st = s->stream;
  for (int j = 0; j < 3; j++) {
    const size_t cnt = d.g1_count[j];
    check_cuda(cudaMemcpyAsync(s->sg1[j].ptr, d.g1_scalars[j], cnt * 32, cudaMemcpyHostToDevice, st), "scalars");
    if (cnt < m) check_cuda(cudaMemsetAsync(s->sg1[j].ptr + 8 * cnt, 0, (m - cnt) * 32, st), "scalar tail");
  }
  check_cuda(cudaMemcpyAsync(s->sg2.ptr, d.g2_scalars, m * 32, cudaMemcpyHostToDevice, st), "scalars");
  for (int j = 0; j < 3; j++)
    check_cuda(cudaMemcpyAsync(s->poly[j].ptr, d.polys[j], N * 32, cudaMemcpyHostToDevice, st), "polynomials");
  if (s->exec) {
    check_cuda(cudaGraphLaunch(s->exec, st), "request graph");
    g_launches.fetch_add(s->graph_kernels, std::memory_order_relaxed);
  } else {
    enqueue_work(s, st, st, st);
  }
  check_cuda(cudaMemcpyAsync(d.out_points, s->results.ptr, (3 * 32 + 64) * 4, cudaMemcpyDeviceToHost, st), "results");
  check_cuda(cudaMemcpyAsync(d.out_h, s->poly[2].ptr, N * 32, cudaMemcpyDeviceToHost, st), "h");
  check_cuda(cudaLaunchHostFunc(st, on_done, r), "completion callback");
}

// Admission. The queue is scanned in order while lanes are free: a request with an idle slot of
// its size is launched at once; one without waits for a busy slot of its size when the size
// already has max(2, reserved) slots (built or being built), and otherwise gets a slot built for
// it by the builder thread when the slot fits the HBM budget (after evicting idle slots of other
// sizes, oldest first); either way the scan goes on, so requests whose slots exist are not held
// up by a slot under construction (measured: a slot built under load took 764 ms, a request of
// the largest size about 120 ms of kernels).
// A request whose slot does not fit stops the scan (later requests wait behind it in FIFO order)
// unless nothing is running, in which case its slot is made anyway.
void Server::dispatcher() {
  cudaSetDevice(ctx->device);
  for (;;) {
    std::vector<std::pair<ServerRequest*, ServerSlot*>> ready;
    std::vector<std::unique_ptr<ServerSlot>> victims;
    bool new_builds = false;
    {
      std::unique_lock<std::mutex> lock(mu);
      for (;;) {
        if (stopping && queue.empty()) return;
        int busy = building;
        for (auto& s : slots) busy += s->busy ? 1 : 0;
        for (auto it = queue.begin(); it != queue.end() && busy < cfg.lanes;) {
          ServerRequest* r = *it;
          const uint32_t log_m = r->desc.log_m;
          ServerSlot* slot = nullptr;
          for (auto& s : slots)
            if (!s->busy && s->log_m == log_m) {
              slot = s.get();
              break;
            }
          if (!slot) {
            uint32_t have = building_of[log_m];
            for (auto& s : slots) have += s->log_m == log_m ? 1 : 0;
            const auto rv = reserved.find(log_m);
            if (have >= std::max<uint32_t>(2, rv == reserved.end() ? 0 : rv->second)) {
              ++it;  // wait for a slot of this size; later requests of other sizes go on
              continue;
            }
            const size_t need = estimate_bytes(log_m);
            for (size_t i = 0; i < slots.size() && bytes_used + need > budget;) {
              if (!slots[i]->busy && slots[i]->log_m != log_m) {
                bytes_used -= std::min(bytes_used, slots[i]->bytes);
                victims.push_back(std::move(slots[i]));
                slots.erase(slots.begin() + i);
                slots_evicted++;
              } else {
                i++;
              }
            }
            if (bytes_used + need > budget && busy > 0) break;  // wait for memory, FIFO from here
            bytes_used += need;
            builds.emplace_back(r, need);
            building++;
            building_of[log_m]++;
            new_builds = true;
          } else {
            slot->busy = true;
            slot->req = r;
            r->slot = slot;
            ready.emplace_back(r, slot);
          }
          r->state = 1;
          r->t_start = now_ms();
          it = queue.erase(it);
          busy++;
        }
        if (!ready.empty() || new_builds || !victims.empty()) break;
        cv.wait(lock);
      }
    }
    if (new_builds) cv.notify_all();
    victims.clear();  // frees device memory outside the lock
    for (auto& rs : ready) {
      try {
        launch(rs.first, rs.second);
      } catch (...) {
        const std::string msg = current_error_text();
        std::lock_guard<std::mutex> lock(mu);
        rs.second->busy = false;
        rs.second->req = nullptr;
        rs.first->state = 3;
        rs.first->error = msg;
        rs.first->t_done = now_ms();
        cv.notify_all();
      }
    }
  }
}

// Makes the slots the dispatcher asked for, one at a time, and launches each waiting request
// on its new slot.
void Server::builder() {
  cudaSetDevice(ctx->device);
  for (;;) {
    std::pair<ServerRequest*, size_t> job;
    {
      std::unique_lock<std::mutex> lock(mu);
      cv.wait(lock, [&] { return !builds.empty() || (stopping && queue.empty() && building == 0); });
      if (builds.empty()) return;
      job = builds.front();
      builds.pop_front();
    }
    ServerRequest* r = job.first;
    ServerSlot* slot = nullptr;
    try {
      const double t0 = now_ms();
      std::unique_ptr<ServerSlot> s = make_slot(r->desc.log_m);
      {
        std::lock_guard<std::mutex> lock(mu);
        build_ms += now_ms() - t0;
        bytes_used = bytes_used - std::min(bytes_used, job.second) + s->bytes;
        slots_created++;
        building--;
        building_of[r->desc.log_m]--;
        s->busy = true;
        s->req = r;
        r->slot = s.get();
        slot = s.get();
        slots.push_back(std::move(s));
      }
      launch(r, slot);
    } catch (...) {
      const std::string msg = current_error_text();
      std::lock_guard<std::mutex> lock(mu);
      if (!slot) {
        bytes_used -= std::min(bytes_used, job.second);
        building--;
        building_of[r->desc.log_m]--;
      } else {
        slot->busy = false;
        slot->req = nullptr;
      }
      r->state = 3;
      r->error = msg;
      r->t_done = now_ms();
    }
    cv.notify_all();
  }
}

// Idle slots of one size made ahead of the requests (so that a burst of requests of that size
// does not wait for slot construction).
void Server::reserve(uint32_t log_m, uint32_t count) {
  if (log_m < 11 || log_m > 26) fail(ZKG_EINVAL, "log_m must be in 11..=26");
  if (!key_for(log_m)) fail(ZKG_EINVAL, "no resident proving key has 2^" + std::to_string(log_m) + " points");
  {
    std::lock_guard<std::mutex> lock(mu);
    reserved[log_m] = std::max(reserved[log_m], count);
  }
  for (;;) {
    size_t need = 0;
    {
      std::lock_guard<std::mutex> lock(mu);
      uint32_t have = 0;
      for (auto& s : slots) have += s->log_m == log_m ? 1 : 0;
      if (have >= count) return;
      need = estimate_bytes(log_m);
      if (bytes_used + need > budget)
        fail(ZKG_ENOMEM, "slot of 2^" + std::to_string(log_m) + " does not fit the HBM budget (" +
                             std::to_string(budget - std::min(budget, bytes_used)) + " bytes left, " +
                             std::to_string(need) + " needed)");
      bytes_used += need;
    }
    std::unique_ptr<ServerSlot> s;
    const double t0 = now_ms();
    try {
      s = make_slot(log_m);
    } catch (...) {
      std::lock_guard<std::mutex> lock(mu);
      bytes_used -= std::min(bytes_used, need);
      throw;
    }
    {
      std::lock_guard<std::mutex> lock(mu);
      build_ms += now_ms() - t0;
      bytes_used = bytes_used - std::min(bytes_used, need) + s->bytes;
      slots_created++;
      slots.push_back(std::move(s));
    }
    cv.notify_all();
  }
}

uint64_t Server::submit(const zkg_proof_request& d) {
  const size_t m = (size_t)1 << d.log_m;
  if (d.log_m < 11 || d.log_m > 26) fail(ZKG_EINVAL, "log_m must be in 11..=26");
  for (int j = 0; j < 3; j++) {
    if (!d.g1_scalars[j] || !d.polys[j]) fail(ZKG_EINVAL, "request input is NULL");
    if (d.g1_count[j] > m || d.g1_count[j] == 0) fail(ZKG_EINVAL, "G1 scalar count must be in 1..=m");
  }
  if (!d.g2_scalars || !d.out_points || !d.out_h) fail(ZKG_EINVAL, "request input is NULL");
  if (!key_for(d.log_m)) fail(ZKG_EINVAL, "no resident proving key has 2^" + std::to_string(d.log_m) + " points");
  std::unique_ptr<ServerRequest> r(new ServerRequest);
  r->desc = d;
  r->server = this;
  r->t_submit = now_ms();
  uint64_t id;
  {
    std::lock_guard<std::mutex> lock(mu);
    id = r->id = next_id++;
    queue.push_back(r.get());
    requests[id] = std::move(r);
  }
  cv.notify_all();
  return id;
}

int Server::wait(uint64_t id, int timeout_ms, zkg_request_times* t) {
  std::unique_lock<std::mutex> lock(mu);
  auto it = requests.find(id);
  if (it == requests.end()) fail(ZKG_EINVAL, "unknown request id");
  ServerRequest* r = it->second.get();
  auto done = [&] { return r->state >= 2; };
  if (timeout_ms < 0) {
    cv.wait(lock, done);
  } else if (!cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), done)) {
    return ZKG_ETIMEDOUT;
  }
  if (t) {
    t->queued_ms = r->t_start - r->t_submit;
    t->device_ms = r->t_done - r->t_start;
    t->total_ms = r->t_done - r->t_submit;
  }
  int state = r->state;
  std::string err = r->error;
  requests.erase(it);
  if (state == 3) fail(ZKG_ECUDA, "request failed: " + err);
  return ZKG_OK;
}

void Server::stats(zkg_server_counters* s) {
  std::lock_guard<std::mutex> lock(mu);
  s->queued = queue.size();
  s->completed = completed;
  s->slots = slots.size();
  s->slots_created = slots_created;
  s->slots_evicted = slots_evicted;
  s->bytes_used = bytes_used;
  s->budget = budget;
  s->build_ms = build_ms;
}

}  // namespace zkg
