// extern "C" entry points of include/zkg.h: argument checks, exception -> status code, and the
// thread-local error message. Every function here is a thin shell over the plans.
#include <cstring>
#include <new>
#include <string>

#include "batch.hpp"
#include "host_curve.hpp"
#include "host_field.hpp"
#include "msm.hpp"
#include "ntt.hpp"
#include "zkey.hpp"
#include "runtime.hpp"
#include "server.hpp"
#include "testing.hpp"
#include "tuning.hpp"

namespace zkg {

std::atomic<uint64_t> g_launches{0};
static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

template <class Fn>
static int guard(Fn&& fn) {
  try {
    fn();
    return ZKG_OK;
  } catch (const Error& e) {
    set_error(e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return ZKG_ENOMEM;
  } catch (...) {
    set_error("unexpected internal error");
    return ZKG_ECUDA;
  }
}

static void need(const void* p, const char* what) {
  if (!p) fail(ZKG_EINVAL, std::string(what) + " is NULL");
}

static zkg_buf* new_buffer(zkg_ctx* ctx, size_t words) {
  zkg_buf* b = new zkg_buf;
  b->ctx = ctx;
  b->words = words;
  try {
    b->ptr = device_alloc(words * 4, "buffer");
  } catch (...) {
    delete b;
    throw;
  }
  return b;
}

static void copy_in(zkg_ctx* ctx, uint32_t* dst, const uint32_t* src, size_t words) {
  if (words == 0) return;
  check_cuda(cudaMemcpyAsync(dst, src, words * 4, cudaMemcpyHostToDevice, ctx->stream), "host to device copy");
  // From pageable memory the copy has consumed the host array when the call returns; from
  // page-locked memory it may still be in flight, so wait for it.
  if (is_pinned(src)) check_cuda(cudaStreamSynchronize(ctx->stream), "host to device copy");
}

}  // namespace zkg

using namespace zkg;

extern "C" {

const char* zkg_last_error(void) { return g_last_error.c_str(); }

int zkg_ctx_new(int device, zkg_ctx** out) {
  return guard([&] {
    need(out, "out");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      fail(ZKG_ENODEV, std::string("no GPU adapter: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device"));
    }
    if (device < 0 || device >= count) fail(ZKG_ENODEV, "no GPU adapter: device index out of range");
    zkg_ctx* ctx = new zkg_ctx;
    ctx->device = device;
    try {
      check_cuda(cudaSetDevice(device), "cudaSetDevice");
      cudaDeviceProp prop;
      check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
      ctx->sm_count = prop.multiProcessorCount;
      std::strncpy(ctx->name, prop.name, sizeof(ctx->name) - 1);
      check_cuda(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
      int least = 0, greatest = 0;
      check_cuda(cudaDeviceGetStreamPriorityRange(&least, &greatest), "cudaDeviceGetStreamPriorityRange");
      check_cuda(cudaStreamCreateWithPriority(&ctx->setup, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
    } catch (...) {
      if (ctx->stream) cudaStreamDestroy(ctx->stream);
      delete ctx;
      throw;
    }
    *out = ctx;
  });
}

void zkg_ctx_free(zkg_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  for (cudaStream_t s : {ctx->up_stream, ctx->down_stream, ctx->setup}) {
    if (!s) continue;
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  delete ctx;
}

int zkg_ctx_sync(zkg_ctx* ctx) {
  return guard([&] {
    need(ctx, "ctx");
    use(ctx);
    check_cuda(cudaStreamSynchronize(ctx->stream), "device work");
    if (ctx->up_stream) check_cuda(cudaStreamSynchronize(ctx->up_stream), "device work");
    if (ctx->down_stream) check_cuda(cudaStreamSynchronize(ctx->down_stream), "device work");
    check_cuda(cudaGetLastError(), "device work");
  });
}

int zkg_ctx_device_name(zkg_ctx* ctx, char* out, size_t cap) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    if (cap == 0) return;
    std::strncpy(out, ctx->name, cap - 1);
    out[cap - 1] = 0;
  });
}

int zkg_buf_new(zkg_ctx* ctx, const uint32_t* data, size_t words, zkg_buf** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    if (words) need(data, "data");
    use(ctx);
    zkg_buf* b = new_buffer(ctx, words);
    try {
      copy_in(ctx, b->ptr, data, words);
    } catch (...) {
      zkg_buf_free(b);
      throw;
    }
    *out = b;
  });
}

int zkg_buf_zeroed(zkg_ctx* ctx, size_t words, zkg_buf** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    use(ctx);
    zkg_buf* b = new_buffer(ctx, words);
    try {
      check_cuda(cudaMemsetAsync(b->ptr, 0, words * 4, ctx->stream), "buffer clear");
    } catch (...) {
      zkg_buf_free(b);
      throw;
    }
    *out = b;
  });
}

int zkg_buf_write(zkg_ctx* ctx, zkg_buf* buf, size_t offset_words, const uint32_t* data, size_t words) {
  return guard([&] {
    need(ctx, "ctx");
    need(buf, "buf");
    if (words) need(data, "data");
    if (offset_words > buf->words || words > buf->words - offset_words)
      fail(ZKG_ESIZE, "write of " + std::to_string(words) + " words at offset " + std::to_string(offset_words) +
                          " overruns a buffer of " + std::to_string(buf->words) + " words");
    use(ctx);
    wait_reads(buf, ctx->stream);
    copy_in(ctx, buf->ptr + offset_words, data, words);
    if (words) mark_use(buf, ctx->stream);
  });
}

int zkg_buf_read(zkg_ctx* ctx, const zkg_buf* buf, uint32_t* out, size_t words) {
  return guard([&] {
    need(ctx, "ctx");
    need(buf, "buf");
    if (words) need(out, "out");
    if (words > buf->words)
      fail(ZKG_ESIZE, "read of " + std::to_string(words) + " words from a buffer of " + std::to_string(buf->words));
    use(ctx);
    if (words)
      check_cuda(cudaMemcpyAsync(out, buf->ptr, words * 4, cudaMemcpyDeviceToHost, ctx->stream), "device to host copy");
    check_cuda(cudaStreamSynchronize(ctx->stream), "GPU read failed");
  });
}

// One-shot event: `waiter` waits for the work queued on `after` so far.
static void order_after(cudaStream_t waiter, cudaStream_t after) {
  cudaEvent_t e;
  check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
  check_cuda(cudaEventRecord(e, after), "cudaEventRecord");
  check_cuda(cudaStreamWaitEvent(waiter, e, 0), "cudaStreamWaitEvent");
  cudaEventDestroy(e);  // released once the wait has been satisfied
}

// Uploads and read-backs on separate streams (the copy engines of the two directions work in
// parallel, and a queued read does not hold back the next step's uploads).
static cudaStream_t side_stream(cudaStream_t* s) {
  if (!*s) check_cuda(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "cudaStreamCreate");
  return *s;
}

int zkg_buf_write_async(zkg_ctx* ctx, zkg_buf* buf, size_t offset_words, const uint32_t* data, size_t words) {
  return guard([&] {
    need(ctx, "ctx");
    need(buf, "buf");
    if (words) need(data, "data");
    if (offset_words > buf->words || words > buf->words - offset_words)
      fail(ZKG_ESIZE, "write of " + std::to_string(words) + " words at offset " + std::to_string(offset_words) +
                          " overruns a buffer of " + std::to_string(buf->words) + " words");
    use(ctx);
    if (!words) return;
    cudaStream_t cs = side_stream(&ctx->up_stream);
    // after the queued work that still uses the buffer; before any work queued from now on
    if (buf->last_use) check_cuda(cudaStreamWaitEvent(cs, buf->last_use, 0), "cudaStreamWaitEvent");
    check_cuda(cudaMemcpyAsync(buf->ptr + offset_words, data, words * 4, cudaMemcpyHostToDevice, cs),
               "host to device copy");
    order_after(ctx->stream, cs);
    mark_use(buf, cs);  // an asynchronous read queued next reads the new data
  });
}

int zkg_buf_read_async(zkg_ctx* ctx, const zkg_buf* buf, uint32_t* out, size_t words) {
  return guard([&] {
    need(ctx, "ctx");
    need(buf, "buf");
    if (words) need(out, "out");
    if (words > buf->words)
      fail(ZKG_ESIZE, "read of " + std::to_string(words) + " words from a buffer of " + std::to_string(buf->words));
    use(ctx);
    if (!words) return;
    cudaStream_t cs = side_stream(&ctx->down_stream);
    // after the data's producer: the buffer's last recorded use (every entry point that queues
    // work on a buffer records one), else all the work queued so far
    if (buf->last_use)
      check_cuda(cudaStreamWaitEvent(cs, buf->last_use, 0), "cudaStreamWaitEvent");
    else
      order_after(cs, ctx->stream);
    check_cuda(cudaMemcpyAsync(out, buf->ptr, words * 4, cudaMemcpyDeviceToHost, cs), "device to host copy");
    // work that writes the buffer later waits for this read; other work runs alongside it
    zkg_buf* m = const_cast<zkg_buf*>(buf);
    if (!m->pending_read)
      check_cuda(cudaEventCreateWithFlags(&m->pending_read, cudaEventDisableTiming), "cudaEventCreate");
    check_cuda(cudaEventRecord(m->pending_read, cs), "cudaEventRecord");
    mark_use(buf, cs);  // and so do later asynchronous writes
  });
}

size_t zkg_buf_words(const zkg_buf* buf) { return buf ? buf->words : 0; }
void* zkg_buf_device_ptr(const zkg_buf* buf) { return buf ? buf->ptr : nullptr; }

void zkg_buf_free(zkg_buf* buf) {
  if (!buf || !buf->owned) return;
  if (buf->ctx) cudaSetDevice(buf->ctx->device);
  if (buf->last_use) cudaEventDestroy(buf->last_use);
  if (buf->pending_read) cudaEventDestroy(buf->pending_read);
  if (buf->ptr) cudaFree(buf->ptr);
  delete buf;
}

uint32_t zkg_msm_default_window(size_t n) { return default_window(n); }

static int upload(zkg_ctx* ctx, const uint32_t* xy, size_t words, bool mont256, zkg_buf** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    if (words) need(xy, "xy");
    if (words % 8) fail(ZKG_EINVAL, "bases hold whole 8-word coordinates");
    use(ctx);
    zkg_buf* b = new_buffer(ctx, words);
    try {
      copy_in(ctx, b->ptr, xy, words);
      upload_bases(ctx, xy, words, mont256, b);
    } catch (...) {
      zkg_buf_free(b);
      throw;
    }
    *out = b;
  });
}

int zkg_msm_upload_bases(zkg_ctx* ctx, const uint32_t* plain_xy, size_t words, zkg_buf** out) {
  return upload(ctx, plain_xy, words, false, out);
}

int zkg_msm_upload_bases_montgomery_256(zkg_ctx* ctx, const uint32_t* xy, size_t words, zkg_buf** out) {
  return upload(ctx, xy, words, true, out);
}

int zkg_zkey_parse(const void* bytes, size_t len, zkg_zkey** out) {
  return guard([&] {
    need(out, "out");
    *out = nullptr;
    std::unique_ptr<zkg_zkey> z(new zkg_zkey);
    z->key = parse_zkey(static_cast<const uint8_t*>(bytes), len);
    *out = z.release();
  });
}

void zkg_zkey_free(zkg_zkey* z) { delete z; }

int zkg_zkey_info(const zkg_zkey* z, zkg_zkey_header* out) {
  return guard([&] {
    need(z, "zkey");
    need(out, "out");
    out->protocol = z->key.protocol;
    out->n_vars = z->key.n_vars;
    out->n_public = z->key.n_public;
    out->domain_size = z->key.domain_size;
  });
}

static const std::vector<uint32_t>& zkey_words(const zkg_zkey* z, uint32_t section) {
  auto it = z->key.points.find(section);
  if (zkey_section_group(section) == 0 || it == z->key.points.end())
    fail(ZKG_EINVAL, "zkey section " + std::to_string(section) + " is not a point section (3, 5, 6, 7, 8, 9)");
  return it->second;
}

int zkg_zkey_points(const zkg_zkey* z, uint32_t section, const uint32_t** words, size_t* points, int* group) {
  return guard([&] {
    need(z, "zkey");
    const std::vector<uint32_t>& w = zkey_words(z, section);
    const int g = zkey_section_group(section);
    if (words) *words = w.data();
    if (points) *points = w.size() / (g == ZKG_G1 ? 16 : 32);
    if (group) *group = g;
  });
}

int zkg_zkey_upload(zkg_ctx* ctx, const zkg_zkey* z, uint32_t section, zkg_buf** out) {
  const zkg_zkey* zz = z;
  const std::vector<uint32_t>* w = nullptr;
  int rc = guard([&] {
    need(zz, "zkey");
    w = &zkey_words(zz, section);
  });
  if (rc != ZKG_OK) return rc;
  return upload(ctx, w->data(), w->size(), true, out);
}

int zkg_msm_new(zkg_ctx* ctx, int group, size_t n, uint32_t c, uint32_t item_points, zkg_msm** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    *out = nullptr;
    *out = new zkg_msm(ctx, group, n, c, item_points);
  });
}

void zkg_msm_free(zkg_msm* msm) {
  if (!msm) return;
  cudaSetDevice(msm->plan.ctx->device);
  cudaStreamSynchronize(msm->plan.ctx->stream);
  delete msm;
}

int zkg_msm_group(const zkg_msm* msm) { return msm ? msm->plan.group : 0; }

int zkg_msm_set_variant(zkg_msm* msm, int variant) {
  return guard([&] {
    need(msm, "msm");
    if (variant < 0 || variant > 6) fail(ZKG_EINVAL, "accumulation variant must be 0..6");
    msm->plan.acc_variant = variant;
  });
}

int zkg_msm_set_sort(zkg_msm* msm, int mode) {
  return guard([&] {
    need(msm, "msm");
    if (mode < 0 || mode > 3) fail(ZKG_EINVAL, "sort aggregation mode must be 0..3");
    msm->plan.sort_agg = mode;
  });
}

int zkg_msm_set_sort_form(zkg_msm* msm, int form) {
  return guard([&] {
    need(msm, "msm");
    if (form < 0 || form > 1) fail(ZKG_EINVAL, "sort form must be 0 or 1");
    msm->plan.sort_form = form;
  });
}

int zkg_msm_fixed_base_table(zkg_ctx* ctx, int group, const zkg_buf* bases, size_t n, uint32_t c, zkg_buf** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(bases, "bases");
    need(out, "out");
    *out = nullptr;
    const uint32_t windows = c >= 1 ? (255 + c - 1) / c : 0;
    const size_t aw = group == ZKG_G2 ? 32 : 16;
    use(ctx);
    zkg_buf* b = new_buffer(ctx, (size_t)windows * n * aw);
    try {
      wait_reads(b, ctx->stream);
      fixed_base_table(ctx, group, bases, n, c, b);
      mark_use(bases, ctx->stream);
      mark_use(b, ctx->stream);
    } catch (...) {
      zkg_buf_free(b);
      throw;
    }
    *out = b;
  });
}

int zkg_msm_set_fixed_base(zkg_msm* msm, int enable) {
  return guard([&] {
    need(msm, "msm");
    msm->plan.set_fixed_base(enable != 0);
  });
}

int zkg_msm_set_glv(zkg_msm* msm, int enable) {
  return guard([&] {
    need(msm, "msm");
    msm->plan.set_glv(enable != 0);
  });
}

int zkg_msm_set_chunk(zkg_msm* msm, size_t points) {
  return guard([&] {
    need(msm, "msm");
    msm->plan.set_chunk(points);
  });
}

int zkg_msm_passes(const zkg_msm* msm, size_t* chunk, size_t* passes) {
  return guard([&] {
    need(msm, "msm");
    if (chunk) *chunk = msm->plan.chunk;
    if (passes) *passes = msm->plan.passes();
  });
}

int zkg_msm_windows(const zkg_msm* msm, uint32_t* windows, int* glv) {
  return guard([&] {
    need(msm, "msm");
    if (windows) *windows = msm->plan.windows;
    if (glv) *glv = msm->plan.glv ? 1 : 0;
  });
}

int zkg_test_glv_split(zkg_ctx* ctx, const uint32_t* scalars, size_t count, uint32_t* out) {
  return guard([&] {
    need(ctx, "ctx");
    need(scalars, "scalars");
    need(out, "out");
    if (count) glv_split(ctx, scalars, count, out);
  });
}

int zkg_msm_params(const zkg_msm* msm, uint32_t* c, uint32_t* item_points, int* variant) {
  return guard([&] {
    need(msm, "msm");
    if (c) *c = msm->plan.c;
    if (item_points) *item_points = msm->plan.seg_len;
    if (variant) *variant = msm->plan.acc_variant;
  });
}

int zkg_msm_run(zkg_msm* msm, const zkg_buf* bases, const zkg_buf* scalars, const zkg_buf** result) {
  return guard([&] {
    need(msm, "msm");
    need(bases, "bases");
    need(scalars, "scalars");
    wait_reads(&msm->plan.result_handle, msm->plan.ctx->stream);
    msm->plan.run(bases, scalars);
    mark_use(bases, msm->plan.ctx->stream);
    mark_use(scalars, msm->plan.ctx->stream);
    mark_use(&msm->plan.result_handle, msm->plan.ctx->stream);
    if (result) *result = &msm->plan.result_handle;
  });
}

int zkg_msm_profile(zkg_msm* msm, const zkg_buf* bases, const zkg_buf* scalars, zkg_stage_time* out, size_t cap,
                    size_t* count) {
  return guard([&] {
    need(msm, "msm");
    need(bases, "bases");
    need(scalars, "scalars");
    wait_reads(&msm->plan.result_handle, msm->plan.ctx->stream);
    auto times = msm->plan.profile(bases, scalars);
    mark_use(&msm->plan.result_handle, msm->plan.ctx->stream);
    size_t k = 0;
    for (auto& t : times) {
      if (k >= cap || !out) break;
      std::memset(out[k].stage, 0, sizeof(out[k].stage));
      std::strncpy(out[k].stage, t.first.c_str(), sizeof(out[k].stage) - 1);
      out[k].ms = t.second;
      k++;
    }
    if (count) *count = k;
  });
}

namespace {
host::U256 word_elem(const uint32_t* w) { return host::from_words32(w); }
void elem_words(const host::U256& e, uint32_t* w) { host::words32(e, w); }
host::U512 word_elem2(const uint32_t* w) { return host::U512{host::from_words32(w), host::from_words32(w + 8)}; }
void elem_words2(const host::U512& e, uint32_t* w) {
  host::words32(e.a, w);
  host::words32(e.b, w + 8);
}
}  // namespace

int zkg_xyzz_add_host(int group, const uint32_t* a, const uint32_t* b, uint32_t* out) {
  return guard([&] {
    need(a, "a");
    need(b, "b");
    need(out, "out");
    if (group == ZKG_G1) {
      using P = host::XyzzH<host::U256>;
      const P pa{word_elem(a), word_elem(a + 8), word_elem(a + 16), word_elem(a + 24)};
      const P pb{word_elem(b), word_elem(b + 8), word_elem(b + 16), word_elem(b + 24)};
      const P r = host::xyzz_add_h(pa, pb);
      elem_words(r.x, out);
      elem_words(r.y, out + 8);
      elem_words(r.zz, out + 16);
      elem_words(r.zzz, out + 24);
    } else if (group == ZKG_G2) {
      using P = host::XyzzH<host::U512>;
      const P pa{word_elem2(a), word_elem2(a + 16), word_elem2(a + 32), word_elem2(a + 48)};
      const P pb{word_elem2(b), word_elem2(b + 16), word_elem2(b + 32), word_elem2(b + 48)};
      const P r = host::xyzz_add_h(pa, pb);
      elem_words2(r.x, out);
      elem_words2(r.y, out + 16);
      elem_words2(r.zz, out + 32);
      elem_words2(r.zzz, out + 48);
    } else {
      fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
    }
  });
}

int zkg_xyzz_to_affine(const uint32_t* words, uint64_t* x, uint64_t* y) {
  if (!words || !x || !y) {
    set_error("NULL argument");
    return -ZKG_EINVAL;
  }
  const host::Field& f = host::fq();
  host::U256 X = host::from_words32(words), Y = host::from_words32(words + 8);
  host::U256 ZZ = host::from_words32(words + 16), ZZZ = host::from_words32(words + 24);
  if (host::is_zero(ZZ)) {
    std::memset(x, 0, 32);
    std::memset(y, 0, 32);
    return 0;
  }
  host::U256 ax = host::from_mont(host::mul(X, host::inverse(ZZ, f), f), f);
  host::U256 ay = host::from_mont(host::mul(Y, host::inverse(ZZZ, f), f), f);
  std::memcpy(x, ax.v, 32);
  std::memcpy(y, ay.v, 32);
  return 1;
}

int zkg_xyzz_to_affine_g2(const uint32_t* words, uint64_t* x, uint64_t* y) {
  if (!words || !x || !y) {
    set_error("NULL argument");
    return -ZKG_EINVAL;
  }
  const host::Field& f = host::fq();
  auto fq2 = [&](int i) { return host::U512{host::from_words32(words + 16 * i), host::from_words32(words + 16 * i + 8)}; };
  host::U512 X = fq2(0), Y = fq2(1), ZZ = fq2(2), ZZZ = fq2(3);
  if (host::is_zero(ZZ.a) && host::is_zero(ZZ.b)) {
    std::memset(x, 0, 64);
    std::memset(y, 0, 64);
    return 0;
  }
  host::U512 ax = host::fq2_mul(X, host::fq2_inverse(ZZ));
  host::U512 ay = host::fq2_mul(Y, host::fq2_inverse(ZZZ));
  host::U256 outs[4] = {host::from_mont(ax.a, f), host::from_mont(ax.b, f), host::from_mont(ay.a, f),
                        host::from_mont(ay.b, f)};
  std::memcpy(x, outs[0].v, 32);
  std::memcpy(x + 4, outs[1].v, 32);
  std::memcpy(y, outs[2].v, 32);
  std::memcpy(y + 4, outs[3].v, 32);
  return 1;
}

int zkg_ntt_new(zkg_ctx* ctx, uint32_t log_n, zkg_ntt** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    *out = nullptr;
    *out = new zkg_ntt(ctx, log_n);
  });
}

void zkg_ntt_free(zkg_ntt* ntt) {
  if (!ntt) return;
  cudaSetDevice(ntt->plan.ctx->device);
  cudaStreamSynchronize(ntt->plan.ctx->stream);
  delete ntt;
}

uint32_t zkg_ntt_log_n(const zkg_ntt* ntt) { return ntt ? ntt->plan.log_n : 0; }

int zkg_ntt_forward(zkg_ntt* ntt, zkg_buf* data) {
  return guard([&] {
    need(ntt, "ntt");
    need(data, "data");
    wait_reads(data, ntt->plan.ctx->stream);
    ntt->plan.run(data, false);
    mark_use(data, ntt->plan.ctx->stream);
  });
}

int zkg_ntt_inverse(zkg_ntt* ntt, zkg_buf* data) {
  return guard([&] {
    need(ntt, "ntt");
    need(data, "data");
    wait_reads(data, ntt->plan.ctx->stream);
    ntt->plan.run(data, true);
    mark_use(data, ntt->plan.ctx->stream);
  });
}

void* zkg_ctx_stream(zkg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

uint64_t zkg_launch_count(void) { return g_launches.load(); }

int zkg_host_alloc(size_t bytes, void** out) {
  return guard([&] {
    need(out, "out");
    *out = nullptr;
    check_cuda(cudaHostAlloc(out, bytes ? bytes : 16, cudaHostAllocDefault), "cudaHostAlloc");
  });
}

void zkg_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

static void write_times(const std::vector<double>& ms, const std::vector<std::string>& names, zkg_stage_time* out,
                        size_t cap, size_t* count) {
  size_t k = 0;
  for (size_t i = 0; i < ms.size() && k < cap && out; i++, k++) {
    std::memset(out[k].stage, 0, sizeof(out[k].stage));
    std::strncpy(out[k].stage, names[i].c_str(), sizeof(out[k].stage) - 1);
    out[k].ms = ms[i];
  }
  if (count) *count = k;
}

int zkg_msm_set_timing(zkg_msm* msm, int enable) {
  return guard([&] {
    need(msm, "msm");
    msm->plan.timer.enabled = enable != 0;
  });
}

int zkg_msm_stage_times(zkg_msm* msm, zkg_stage_time* out, size_t cap, size_t* count, size_t* runs) {
  return guard([&] {
    need(msm, "msm");
    use(msm->plan.ctx);
    std::vector<double> ms = msm->plan.timer.collect(MsmPlan::kStages, runs);
    std::vector<std::string> names;
    for (int i = 0; i < MsmPlan::kStages; i++) names.push_back(MsmPlan::stage_name(i));
    write_times(ms, names, out, cap, count);
  });
}

int zkg_msm_last_entries(zkg_msm* msm, uint64_t* entries) {
  return guard([&] {
    need(msm, "msm");
    need(entries, "entries");
    use(msm->plan.ctx);
    uint32_t v = 0;
    check_cuda(cudaMemcpyAsync(&v, msm->plan.slot_start.ptr + msm->plan.slots, 4, cudaMemcpyDeviceToHost,
                               msm->plan.ctx->stream),
               "entry count");
    check_cuda(cudaStreamSynchronize(msm->plan.ctx->stream), "entry count");
    *entries = v;
  });
}

int zkg_ntt_set_timing(zkg_ntt* ntt, int enable) {
  return guard([&] {
    need(ntt, "ntt");
    ntt->plan.timer.enabled = enable != 0;
  });
}

int zkg_ntt_pass_times(zkg_ntt* ntt, zkg_stage_time* out, size_t cap, size_t* count, size_t* runs) {
  return guard([&] {
    need(ntt, "ntt");
    use(ntt->plan.ctx);
    int np = (int)ntt->plan.passes.size();
    std::vector<double> ms = ntt->plan.timer.collect(np, runs);
    std::vector<std::string> names;
    for (int i = 0; i < np; i++) names.push_back("pass " + std::to_string(i));
    write_times(ms, names, out, cap, count);
  });
}

int zkg_bench_integer_pipe(zkg_ctx* ctx, int variant, double* ops_per_second) {
  return guard([&] {
    need(ctx, "ctx");
    need(ops_per_second, "ops_per_second");
    *ops_per_second = bench_integer_pipe(ctx, variant);
  });
}

int zkg_coset_new(zkg_ctx* ctx, uint32_t log_n, const uint32_t* g, zkg_coset** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(g, "g");
    need(out, "out");
    *out = nullptr;
    *out = new zkg_coset(ctx, log_n, g);
  });
}

void zkg_coset_free(zkg_coset* c) {
  if (!c) return;
  cudaSetDevice(c->shift.ctx->device);
  cudaStreamSynchronize(c->shift.ctx->stream);
  delete c;
}

int zkg_coset_shift(zkg_coset* c, zkg_buf* data) {
  return guard([&] {
    need(c, "coset");
    need(data, "data");
    wait_reads(data, c->shift.ctx->stream);
    c->shift.run(data);
    mark_use(data, c->shift.ctx->stream);
  });
}

int zkg_ntt_inverse_coset(zkg_ntt* ntt, zkg_buf* data, zkg_coset* c) {
  return guard([&] {
    need(ntt, "ntt");
    need(data, "data");
    need(c, "coset");
    wait_reads(data, ntt->plan.ctx->stream);
    ntt->plan.run(data, true, &c->shift);
    mark_use(data, ntt->plan.ctx->stream);
  });
}

static void need_elements(const zkg_buf* b, uint32_t log_n, const char* what) {
  const size_t need_w = (size_t)8 << log_n;
  if (b->words < need_w)
    zkg::fail(ZKG_ESIZE, std::string(what) + " buffer holds " + std::to_string(b->words * 4) + " bytes; 2^" +
                             std::to_string(log_n) + " elements need " + std::to_string(need_w * 4));
}

int zkg_quotient(zkg_ctx* ctx, zkg_buf* a, const zkg_buf* b, const zkg_buf* c, uint32_t log_n, const uint32_t* g) {
  return guard([&] {
    need(ctx, "ctx");
    need(a, "a");
    need(b, "b");
    need(c, "c");
    need(g, "g");
    if (log_n < 1 || log_n > 28) fail(ZKG_EINVAL, "log_n must be in 1..=28");
    need_elements(a, log_n, "a");
    need_elements(b, log_n, "b");
    need_elements(c, log_n, "c");
    const host::U256 zinv = coset_zinv(g, log_n);
    use(ctx);
    wait_reads(a, ctx->stream);
    quotient(a->ptr, a->ptr, b->ptr, c->ptr, log_n, zinv, ctx->stream);
    mark_use(a, ctx->stream);
    mark_use(b, ctx->stream);
    mark_use(c, ctx->stream);
  });
}

int zkg_ntt_forward_quotient(zkg_ntt* ntt, zkg_buf* data, const zkg_buf* a, const zkg_buf* b, const uint32_t* g) {
  return guard([&] {
    need(ntt, "ntt");
    need(data, "data");
    need(a, "a");
    need(b, "b");
    need(g, "g");
    const uint32_t log_n = ntt->plan.log_n;
    need_elements(a, log_n, "a");
    need_elements(b, log_n, "b");
    const Quotient q{a->ptr, b->ptr, coset_zinv(g, log_n)};
    cudaStream_t s = ntt->plan.ctx->stream;
    wait_reads(data, s);
    ntt->plan.run(data, false, nullptr, &q);
    mark_use(data, s);
    mark_use(a, s);
    mark_use(b, s);
  });
}

int zkg_batch_new(zkg_ctx* ctx, zkg_batch** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(out, "out");
    *out = nullptr;
    *out = new zkg_batch(ctx);
  });
}

void zkg_batch_free(zkg_batch* b) {
  if (!b) return;
  cudaSetDevice(b->batch.ctx->device);
  cudaStreamSynchronize(b->batch.ctx->stream);
  delete b;
}

int zkg_batch_add_msm(zkg_batch* b, zkg_msm* msm, const zkg_buf* bases, const zkg_buf* scalars, zkg_buf* result,
                      int lane) {
  return guard([&] {
    need(b, "batch");
    need(msm, "msm");
    need(bases, "bases");
    need(scalars, "scalars");
    b->batch.add_msm(&msm->plan, bases, scalars, result, lane);
  });
}

int zkg_batch_add_ntt(zkg_batch* b, zkg_ntt* ntt, zkg_buf* data, int inverse, int lane) {
  return guard([&] {
    need(b, "batch");
    need(ntt, "ntt");
    need(data, "data");
    b->batch.add_ntt(&ntt->plan, data, inverse != 0, lane);
  });
}

int zkg_batch_add_coset(zkg_batch* b, zkg_coset* c, zkg_buf* data, int lane) {
  return guard([&] {
    need(b, "batch");
    need(c, "coset");
    need(data, "data");
    b->batch.add_coset(&c->shift, data, lane);
  });
}

int zkg_batch_capture(zkg_batch* b) {
  return guard([&] {
    need(b, "batch");
    b->batch.capture();
  });
}

int zkg_batch_launch(zkg_batch* b) {
  return guard([&] {
    need(b, "batch");
    b->batch.launch();
  });
}

int zkg_batch_run_streams(zkg_batch* b) {
  return guard([&] {
    need(b, "batch");
    b->batch.run_streams();
  });
}

size_t zkg_batch_kernels(const zkg_batch* b) { return b ? b->batch.kernels_per_launch() : 0; }

int zkg_server_new(zkg_ctx* ctx, const zkg_server_config* config, zkg_server** out) {
  return guard([&] {
    need(ctx, "ctx");
    need(config, "config");
    need(out, "out");
    *out = nullptr;
    *out = new zkg_server(ctx, *config);
  });
}

void zkg_server_free(zkg_server* s) { delete s; }

int zkg_server_add_key(zkg_server* s, size_t n, const zkg_buf* g1, const zkg_buf* g2) {
  return guard([&] {
    need(s, "server");
    need(g1, "g1_bases");
    need(g2, "g2_bases");
    s->server.add_key(n, g1, g2);
  });
}

int zkg_server_submit(zkg_server* s, const zkg_proof_request* r, uint64_t* id) {
  return guard([&] {
    need(s, "server");
    need(r, "request");
    need(id, "id");
    *id = s->server.submit(*r);
  });
}

int zkg_server_wait(zkg_server* s, uint64_t id, int timeout_ms, zkg_request_times* times) {
  int rc = ZKG_OK;
  int g = guard([&] {
    need(s, "server");
    rc = s->server.wait(id, timeout_ms, times);
  });
  if (g != ZKG_OK) return g;
  if (rc == ZKG_ETIMEDOUT) set_error("request not done within the timeout");
  return rc;
}

int zkg_server_stats(zkg_server* s, zkg_server_counters* st) {
  return guard([&] {
    need(s, "server");
    need(st, "stats");
    s->server.stats(st);
  });
}

int zkg_server_reserve(zkg_server* s, uint32_t log_m, uint32_t count) {
  return guard([&] {
    need(s, "server");
    s->server.reserve(log_m, count);
  });
}

int zkg_tune_msm(zkg_ctx* ctx, int group, size_t n, const zkg_buf* bases, const zkg_buf* scalars, int reps,
                 zkg_msm_tuning* out, size_t cap, size_t* count) {
  return guard([&] {
    need(ctx, "ctx");
    need(bases, "bases");
    need(scalars, "scalars");
    if (group != ZKG_G1 && group != ZKG_G2) fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
    if (n < 1) fail(ZKG_EINVAL, "an MSM needs at least one point");
    auto all = tune_msm(ctx, group, n, bases, scalars, reps < 1 ? 1 : reps);
    size_t k = 0;
    for (; k < all.size() && k < cap && out; k++) out[k] = all[k];
    if (count) *count = k;
  });
}

int zkg_ntt_set_variant(zkg_ntt* ntt, int variant) {
  return guard([&] {
    need(ntt, "ntt");
    if (!ntt->plan.set_variant(variant)) fail(ZKG_EINVAL, "NTT variant must be 0..4");
  });
}

int zkg_ntt_set_max_stages(zkg_ntt* ntt, uint32_t max_stages) {
  return guard([&] {
    need(ntt, "ntt");
    if (!ntt->plan.set_max_stages(max_stages))
      fail(ZKG_EINVAL, "max_stages must be in 6..=" + std::to_string(ntt->plan.tile_log()) + " for this NTT variant");
  });
}

int zkg_ntt_params(const zkg_ntt* ntt, int* variant, uint32_t* max_stages, uint32_t* passes) {
  return guard([&] {
    need(ntt, "ntt");
    if (variant) *variant = ntt->plan.variant;
    if (max_stages) *max_stages = ntt->plan.max_stages;
    if (passes) *passes = (uint32_t)ntt->plan.passes.size();
  });
}

int zkg_tune_ntt(zkg_ctx* ctx, uint32_t log_n, zkg_buf* data, int reps, int* best_variant, uint32_t* best_max_stages,
                 double* best_ms) {
  return guard([&] {
    need(ctx, "ctx");
    need(data, "data");
    use(ctx);
    wait_reads(data, ctx->stream);
    auto all = tune_ntt(ctx, log_n, data, reps < 1 ? 1 : reps);
    mark_use(data, ctx->stream);
    if (all.empty()) fail(ZKG_EINVAL, "no pass split applies to this size");
    if (best_variant) *best_variant = all[0].variant;
    if (best_max_stages) *best_max_stages = all[0].max_stages;
    if (best_ms) *best_ms = all[0].ms;
  });
}

int zkg_test_point_ops(zkg_ctx* ctx, int group, const uint32_t* pairs, size_t count, uint32_t* out) {
  return guard([&] {
    need(ctx, "ctx");
    need(pairs, "pairs");
    need(out, "out");
    if (group != ZKG_G1 && group != ZKG_G2) fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
    if (count) point_ops(ctx, group, pairs, count, out);
  });
}

int zkg_generator_multiples(zkg_ctx* ctx, int group, const zkg_buf* scalars, size_t n, int mont256, zkg_buf* out) {
  return guard([&] {
    need(ctx, "ctx");
    need(scalars, "scalars");
    need(out, "out");
    if (group != ZKG_G1 && group != ZKG_G2) fail(ZKG_EINVAL, "group must be ZKG_G1 or ZKG_G2");
    use(ctx);
    wait_reads(out, ctx->stream);
    if (n) generator_multiples(ctx, group, scalars, n, mont256, out);
    mark_use(out, ctx->stream);
    mark_use(scalars, ctx->stream);
  });
}

}  // extern "C"
