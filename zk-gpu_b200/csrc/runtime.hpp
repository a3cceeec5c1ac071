// Device runtime behind the C-ABI: one context per GPU with one ordered CUDA stream, device
// buffers of u32 words, and status codes with a thread-local error message.
//
// Replaces the reference's wgpu wrapper (src/gpu.rs:6-199): Gpu{device, queue} becomes a
// CUDA device plus a non-blocking stream (all work is ordered on it and asynchronous until a
// read or a wait, like the wgpu queue); Gpu::buffer / empty_buffer become cudaMalloc'd word
// buffers; Gpu::read is a blocking device-to-host copy; report_errors / try_read_async become
// status codes plus zkg_last_error(). Pipelines, bind groups and WGSL compilation have no
// counterpart: kernels are compiled ahead of time for sm_100a.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/zkg.h"

namespace zkg {

void set_error(const std::string& msg);
const std::string& last_error();

// Thrown inside the library, turned into a status code at the C-ABI boundary.
struct Error {
  int code;
  std::string msg;
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error{code, msg}; }

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? ZKG_ENOMEM : ZKG_ECUDA;
    fail(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

// Kernels launched by this library in this process (zkg_launch_count).
extern std::atomic<uint64_t> g_launches;

// Checks the launch that was just made (configuration errors surface here; faults surface at
// the next synchronising call) and counts it.
inline void check_launch(const char* kernel) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  check_cuda(cudaGetLastError(), kernel);
}

}  // namespace zkg

struct zkg_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;       // every kernel of the context
  cudaStream_t up_stream = nullptr;    // asynchronous buffer writes (created on first use)
  cudaStream_t down_stream = nullptr;  // asynchronous buffer reads (created on first use)
  // One-time set-up work of plans (twiddle and power tables), waited for by the constructor.
  // Highest stream priority: the hardware hands its blocks out before those of kernels already
  // queued, so a plan made while the device is busy (a server slot made under load) does not
  // wait for all of that work.
  cudaStream_t setup = nullptr;
  int sm_count = 0;
  char name[256] = {0};
};

struct zkg_buf {
  zkg_ctx* ctx = nullptr;
  uint32_t* ptr = nullptr;
  size_t words = 0;
  bool owned = true;  // false for plan-owned results handed out as borrowed handles
  // Recorded after the last queued work that uses the buffer (a kernel on the context stream,
  // an asynchronous read or write): an asynchronous write waits for it, and so does an
  // asynchronous read (the data's producer is the last use before it). Created on first use.
  cudaEvent_t last_use = nullptr;
  // Recorded after the last asynchronous read: work that writes the buffer waits for it, other
  // work does not (a read-back overlaps the kernels queued after it).
  cudaEvent_t pending_read = nullptr;
};

namespace zkg {

// Makes the context's device current for this thread.
inline void use(zkg_ctx* ctx) { check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice"); }

// Notes that work queued on `stream` so far uses `b` (later asynchronous writes wait for it).
inline void mark_use(const zkg_buf* b, cudaStream_t stream) {
  if (!b) return;
  zkg_buf* m = const_cast<zkg_buf*>(b);
  if (!m->last_use) check_cuda(cudaEventCreateWithFlags(&m->last_use, cudaEventDisableTiming), "cudaEventCreate");
  check_cuda(cudaEventRecord(m->last_use, stream), "cudaEventRecord");
}

// Work about to be queued on `stream` writes `b`: it waits for the queued asynchronous reads of b.
inline void wait_reads(const zkg_buf* b, cudaStream_t stream) {
  if (b && b->pending_read) check_cuda(cudaStreamWaitEvent(stream, b->pending_read, 0), "cudaStreamWaitEvent");
}

inline uint32_t* device_alloc(size_t bytes, const char* what) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  check_cuda(cudaMalloc(&p, bytes), what);
  return static_cast<uint32_t*>(p);
}

// Owns a device allocation; frees it on destruction.
struct DeviceArray {
  uint32_t* ptr = nullptr;
  size_t words = 0;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  ~DeviceArray() { release(); }
  void alloc(size_t w, const char* what) {
    release();
    ptr = device_alloc(w * 4, what);
    words = w;
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    words = 0;
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(ptr);
  }
};

// True when the host pointer is page-locked (an async copy from it may still be in flight
// after the call returns, so the copy must be waited for before returning to the caller).
inline bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Device time per named stage, summed over runs, from CUDA events recorded on the launching
// stream while enabled (no synchronisation until collect()).
struct StageTimer {
  bool enabled = false;
  size_t runs = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> pool;

  ~StageTimer() {
    for (auto& p : pending) {
      pool.push_back(p.second.first);
      pool.push_back(p.second.second);
    }
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    check_cuda(cudaEventCreate(&e), "cudaEventCreate");
    return e;
  }
  // Records the start of stage `id`; returns the index to pass to end().
  size_t begin(int id, cudaStream_t s) {
    cudaEvent_t a = take(), b = take();
    check_cuda(cudaEventRecord(a, s), "cudaEventRecord");
    pending.push_back({id, {a, b}});
    return pending.size() - 1;
  }
  void end(size_t idx, cudaStream_t s) { check_cuda(cudaEventRecord(pending[idx].second.second, s), "cudaEventRecord"); }
  // Waits for the recorded events and returns summed milliseconds per stage id.
  std::vector<double> collect(int stages, size_t* out_runs) {
    std::vector<double> ms(stages, 0.0);
    for (auto& p : pending) {
      check_cuda(cudaEventSynchronize(p.second.second), "stage timing");
      float t = 0;
      check_cuda(cudaEventElapsedTime(&t, p.second.first, p.second.second), "cudaEventElapsedTime");
      if (p.first >= 0 && p.first < stages) ms[p.first] += t;
      pool.push_back(p.second.first);
      pool.push_back(p.second.second);
    }
    pending.clear();
    if (out_runs) *out_runs = runs;
    runs = 0;
    return ms;
  }
};

inline unsigned grid_for(size_t threads, unsigned block) {
  size_t g = (threads + block - 1) / block;
  return (unsigned)(g == 0 ? 1 : g);
}

}  // namespace zkg
