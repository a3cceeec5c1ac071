// Set-up and test kernels: the curve point-op check (the reference's tests/curve.rs:22-44 WGSL
// kernel) and a fixed-base batch multiplication [k_i]G that builds proving-key-like bases on
// the device (the reference builds them with arkworks on the host, tests/g2.rs:320-333).
#include <vector>

#include "curve.cuh"
#include "field_f64.cuh"
#include "host_field.hpp"
#include "runtime.hpp"
#include "testing.hpp"

namespace zkg {

__device__ __forceinline__ Fq from_mont(const Fq& a) {
  Fq one_plain = Fq::zero();
  one_plain.w[0] = 1;
  return a * one_plain;
}
__device__ __forceinline__ Fq2 from_mont(const Fq2& a) { return Fq2{from_mont(a.a), from_mont(a.b)}; }

// ------------------------------------------------------------------ point ops test

template <class F>
__global__ void point_ops_kernel(const uint32_t* __restrict__ pairs, size_t count, uint32_t* __restrict__ out) {
  constexpr int W = FieldWords<F>::value;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  Affine<F> p = load_affine<F>(pairs + i * 4 * W);
  Affine<F> q = load_affine<F>(pairs + i * 4 * W + 2 * W);
  Xyzz<F> sum = xyzz_add_affine(from_affine(p), q);
  Xyzz<F> dbl = xyzz_double(from_affine(p));
  Xyzz<F> both = xyzz_add(sum, dbl);
  uint32_t* o = out + i * 12 * W;
  store_xyzz(o, sum);
  store_xyzz(o + 4 * W, dbl);
  store_xyzz(o + 8 * W, both);
}

void point_ops(zkg_ctx* ctx, int group, const uint32_t* pairs, size_t count, uint32_t* out) {
  use(ctx);
  const size_t w = group == ZKG_G1 ? 8 : 16;
  DeviceArray in, res;
  in.alloc(count * 4 * w, "point ops input");
  res.alloc(count * 12 * w, "point ops output");
  check_cuda(cudaMemcpyAsync(in.ptr, pairs, count * 4 * w * 4, cudaMemcpyHostToDevice, ctx->stream), "copy");
  if (group == ZKG_G1)
    point_ops_kernel<Fq><<<grid_for(count, 64), 64, 0, ctx->stream>>>(in.ptr, count, res.ptr);
  else
    point_ops_kernel<Fq2><<<grid_for(count, 64), 64, 0, ctx->stream>>>(in.ptr, count, res.ptr);
  check_launch("point_ops_kernel");
  check_cuda(cudaMemcpyAsync(out, res.ptr, count * 12 * w * 4, cudaMemcpyDeviceToHost, ctx->stream), "copy");
  check_cuda(cudaStreamSynchronize(ctx->stream), "point ops");
}

// ------------------------------------------------------------------ generator multiples

// Table entry (j, d) = [d * 2^(8j)] G, affine Montgomery form; entry d = 0 is infinity.
template <class F>
__global__ void comb_table_kernel(Affine<F> gen, uint32_t* __restrict__ table) {
  constexpr int AW = 2 * FieldWords<F>::value;
  uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= 32 * 256) return;
  uint32_t j = id >> 8, d = id & 255;
  Xyzz<F> acc = xyzz_infinity<F>();
  for (int bit = 7; bit >= 0; bit--) {
    acc = xyzz_double(acc);
    if ((d >> bit) & 1) acc = xyzz_add_affine(acc, gen);
  }
  for (uint32_t k = 0; k < 8 * j; k++) acc = xyzz_double(acc);
  Affine<F> a = to_affine(acc);
  store_elem(table + (size_t)id * AW, a.x);
  store_elem(table + (size_t)id * AW + AW / 2, a.y);
}

template <class F>
__global__ void generator_multiples_kernel(const uint32_t* __restrict__ table, const uint32_t* __restrict__ k, size_t n,
                                           int mont256, uint32_t* __restrict__ out) {
  constexpr int AW = 2 * FieldWords<F>::value;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Xyzz<F> acc = xyzz_infinity<F>();
  for (int word = 0; word < 8; word++) {
    uint32_t v = __ldg(&k[8 * i + word]);
    for (int b = 0; b < 4; b++) {
      uint32_t d = (v >> (8 * b)) & 255;
      if (d) acc = xyzz_add_affine(acc, load_affine<F>(table + (size_t)((4 * word + b) * 256 + d) * AW));
    }
  }
  Affine<F> a = to_affine(acc);
  if (!mont256) {
    a.x = from_mont(a.x);
    a.y = from_mont(a.y);
  }
  store_elem(out + i * AW, a.x);
  store_elem(out + i * AW + AW / 2, a.y);
}

// Standard BN254 G2 generator, plain coordinates x.a, x.b, y.a, y.b (8 LE words each).
static const uint32_t kG2Gen[32] = {
    0xd992f6ed, 0x46debd5c, 0xf75edadd, 0x674322d4, 0x5e5c4479, 0x426a0066, 0x121f1e76, 0x1800deef,
    0xaef312c2, 0x97e485b7, 0x35a9e712, 0xf1aa4933, 0x31fb5d25, 0x7260bfb7, 0x920d483a, 0x198e9393,
    0x66fa7daa, 0x4ce6cc01, 0x0c43d37b, 0xe3d1e769, 0x8dcb408f, 0x4aab7180, 0xdb8c6deb, 0x12c85ea5,
    0xd122975b, 0x55acdadc, 0x70b38ef3, 0xbc4b3133, 0x690c3395, 0xec9e99ad, 0x585ff075, 0x090689d0,
};

static Fq host_mont(const uint32_t* plain) {
  Fq r;
  host::words32(host::to_mont(host::from_words32(plain), host::fq()), r.w);
  return r;
}

void generator_multiples(zkg_ctx* ctx, int group, const zkg_buf* scalars, size_t n, int mont256, zkg_buf* out) {
  const size_t aw = group == ZKG_G1 ? 16 : 32;
  if (scalars->words < 8 * n) fail(ZKG_ESIZE, "scalars buffer too small for n scalars");
  if (out->words < aw * n) fail(ZKG_ESIZE, "output buffer too small for n points");
  use(ctx);
  DeviceArray table;
  table.alloc(32 * 256 * aw, "comb table");
  if (group == ZKG_G1) {
    uint32_t one[8] = {1, 0, 0, 0, 0, 0, 0, 0}, two[8] = {2, 0, 0, 0, 0, 0, 0, 0};
    Affine<Fq> g{host_mont(one), host_mont(two)};
    comb_table_kernel<Fq><<<32, 256, 0, ctx->stream>>>(g, table.ptr);
    check_launch("comb_table_kernel");
    generator_multiples_kernel<Fq><<<grid_for(n, 128), 128, 0, ctx->stream>>>(table.ptr, scalars->ptr, n, mont256,
                                                                              out->ptr);
  } else {
    Affine<Fq2> g{Fq2{host_mont(kG2Gen), host_mont(kG2Gen + 8)}, Fq2{host_mont(kG2Gen + 16), host_mont(kG2Gen + 24)}};
    comb_table_kernel<Fq2><<<32, 256, 0, ctx->stream>>>(g, table.ptr);
    check_launch("comb_table_kernel");
    generator_multiples_kernel<Fq2><<<grid_for(n, 128), 128, 0, ctx->stream>>>(table.ptr, scalars->ptr, n, mont256,
                                                                               out->ptr);
  }
  check_launch("generator_multiples_kernel");
  // The table is freed on return: finish the kernels that read it.
  check_cuda(cudaStreamSynchronize(ctx->stream), "generator multiples");
}

// ------------------------------------------------------------------ roofline denominators
//
// Peak rates measured on the running GPU, the denominators of the bench line's fractions:
// variant 0: mad.lo.u32, 1: mad.hi.u32, 2: a carry chain of mad.lo.cc / madc.hi.cc as in the
// Montgomery rows (8 multiply-adds per step each), 3: Fq Montgomery products in the library's
// integer form, 9: fma.rn.f64, 11: Fq products in the double-precision limb form (checked
// equal to the integer form on the device before it is timed).

// Eight independent multiply-add chains per thread (enough independent work to keep the pipe
// full at any occupancy).
template <int V>
__global__ void imad_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
  uint32_t a[8];
#pragma unroll
  for (int j = 0; j < 8; j++) a[j] = (threadIdx.x + 977u * j) ^ seed;
  const uint32_t b = seed | 1u;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if (V == 0) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(b), "r"(a[(j + 1) & 7]));
      if (V == 1) asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(b), "r"(a[(j + 1) & 7]));
    }
    if (V == 2)
      asm volatile(
          "mad.lo.cc.u32  %0, %0, %8, %1;\n\t"
          "madc.hi.cc.u32 %1, %1, %8, %2;\n\t"
          "madc.lo.cc.u32 %2, %2, %8, %3;\n\t"
          "madc.hi.cc.u32 %3, %3, %8, %4;\n\t"
          "madc.lo.cc.u32 %4, %4, %8, %5;\n\t"
          "madc.hi.cc.u32 %5, %5, %8, %6;\n\t"
          "madc.lo.cc.u32 %6, %6, %8, %7;\n\t"
          "madc.hi.u32    %7, %7, %8, %0;"
          : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
          : "r"(b));
  }
  uint32_t x = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) x ^= a[j];
  if (x == 0x9e3779b9u) out[0] = x;  // keeps the chains live
}

// FP64 pipe throughput: eight independent fma.rn.f64 chains. Values stay normal (b < 1, c > 0).
__global__ void dfma_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
  double d[8];
#pragma unroll
  for (int j = 0; j < 8; j++) d[j] = 1.0 + 1e-3 * (double)((threadIdx.x + 31u * j + seed) & 1023u);
  const double b = 0.9999999, c = 1e-3;
  for (uint32_t it = 0; it < iters; it++) {
#pragma unroll
    for (int j = 0; j < 8; j++) asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(d[j]) : "d"(b), "d"(c));
  }
  double s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += d[j];
  if (s == 12345.0) out[0] = 1;  // keeps the chains live
}

// Fq Montgomery products per second (the reference's examples/field_bench.rs idea).
__global__ void mulmod_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
  Fq x = Fq::one(), y = Fq::one();
  x.w[0] ^= threadIdx.x + seed;
  y.w[1] ^= blockIdx.x;
  Fq z = x;
  for (uint32_t it = 0; it < iters; it++) {
    x = x * y;
    z = z * y;
  }
  if ((x.w[0] ^ z.w[3]) == 0x9e3779b9u) out[0] = x.w[0];
}

// Fq products on the double-precision pipe (field_f64.cuh), same loop as mulmod_kernel.
__global__ void mulmod_f64_kernel(uint32_t* out, uint32_t iters, uint32_t seed) {
  double x[5], y[5], z[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    const uint64_t m = k < 4 ? f64::kM52 : 0xffffffffull;
    x[k] = f64::limb_to_double(((uint64_t)(threadIdx.x + seed) * 0x9e3779b97f4a7c15ull >> (7 * k)) & m);
    y[k] = f64::limb_to_double(((uint64_t)(blockIdx.x + 977u * k) * 0xd1b54a32d192ed03ull) & m);
    z[k] = y[k];
  }
  for (uint32_t it = 0; it < iters; it++) {
    f64::mont_mul<f64::FqLimbs>(x, y, x);
    f64::mont_mul<f64::FqLimbs>(z, y, z);
  }
  if (x[0] == z[3] + 0.5) out[0] = (uint32_t)x[1];  // keeps the chains live
}

// 16 a mod p for a canonical Fq value: the factor between Montgomery forms with R = 2^256 and
// R = 2^260 of the same element.
__device__ __forceinline__ Fq times16(Fq a) {
#pragma unroll
  for (int i = 0; i < 4; i++) a = a + a;
  return a;
}

// Counts threads whose double-precision product chain differs from the integer chain.
__global__ void mulmod_f64_compare_kernel(uint32_t* mismatches, uint32_t iters) {
  Fq x = Fq::one(), y = Fq::one();
  x.w[0] ^= threadIdx.x * 2654435761u + blockIdx.x;
  x.w[7] &= 0x0fffffffu;
  y.w[2] ^= blockIdx.x * 40503u + 7u;
  y.w[7] &= 0x0fffffffu;
  if (threadIdx.x == 0) x = Fq::zero();
  Fq xs = times16(x), ys = times16(y);
  double a[5], b[5];
  f64::words_to_limbs(xs.w, a);
  f64::words_to_limbs(ys.w, b);
  Fq u = x;
  for (uint32_t it = 0; it < iters; it++) {
    u = u * y;
    f64::mont_mul<f64::FqLimbs>(a, b, a);
  }
  uint32_t w[8];
  f64::limbs_to_words(a, w);
  const Fq want = times16(u);
  // a is below 2p: it must equal want or want + p
  const uint32_t pw[8] = {FqParams::P0, FqParams::P1, FqParams::P2, FqParams::P3,
                          FqParams::P4, FqParams::P5, FqParams::P6, FqParams::P7};
  bool same = true, same_p = true;
  uint64_t carry = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    same = same && w[i] == want.w[i];
    const uint64_t t = (uint64_t)want.w[i] + pw[i] + carry;
    carry = t >> 32;
    same_p = same_p && w[i] == (uint32_t)t;
  }
  if (!same && !same_p) atomicAdd(mismatches, 1u);
}

bool integer_pipe_variant_known(int variant) {
  return variant == 0 || variant == 1 || variant == 2 || variant == 3 || variant == 9 || variant == 11;
}

double bench_integer_pipe(zkg_ctx* ctx, int variant) {
  if (!integer_pipe_variant_known(variant)) fail(ZKG_EINVAL, "variant must be one of 0, 1, 2, 3, 9, 11");
  use(ctx);
  DeviceArray sink;
  sink.alloc(16, "sink");
  const unsigned blocks = (unsigned)ctx->sm_count * 8, threads = 256;
  const bool product = variant == 3 || variant == 11;
  const uint32_t iters = product ? 256 : 4096;
  if (variant == 11) {  // the limb form must agree with the integer product first
    check_cuda(cudaMemsetAsync(sink.ptr, 0, 4, ctx->stream), "clear");
    mulmod_f64_compare_kernel<<<blocks, threads, 0, ctx->stream>>>(sink.ptr, 64);
    check_launch("mulmod_f64_compare_kernel");
    uint32_t bad = 0;
    check_cuda(cudaMemcpyAsync(&bad, sink.ptr, 4, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    check_cuda(cudaStreamSynchronize(ctx->stream), "compare");
    if (bad) fail(ZKG_ECUDA, "the double-precision product differs from the integer one in " + std::to_string(bad) + " threads");
  }
  cudaEvent_t a, b;
  check_cuda(cudaEventCreate(&a), "event");
  check_cuda(cudaEventCreate(&b), "event");
  auto launch = [&] {
    switch (variant) {
      case 0: imad_kernel<0><<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
      case 1: imad_kernel<1><<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
      case 2: imad_kernel<2><<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
      case 9: dfma_kernel<<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
      case 11: mulmod_f64_kernel<<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
      default: mulmod_kernel<<<blocks, threads, 0, ctx->stream>>>(sink.ptr, iters, 12345u); break;
    }
    check_launch("integer pipe benchmark");
  };
  launch();  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; rep++) {
    check_cuda(cudaEventRecord(a, ctx->stream), "event");
    launch();
    check_cuda(cudaEventRecord(b, ctx->stream), "event");
    check_cuda(cudaEventSynchronize(b), "integer pipe benchmark");
    float ms = 0;
    check_cuda(cudaEventElapsedTime(&ms, a, b), "event");
    if (ms < best) best = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  double threads_total = (double)blocks * threads;
  // variants 0-2 and 9: 8 multiply-adds (or FMAs) per step; 3 and 11: 2 Fq products per step.
  double per = product ? 2.0 : 8.0;
  double ops = threads_total * iters * per;
  return ops / (best * 1e-3);
}

}  // namespace zkg
