// NTT plan (host side of Ntt, src/ntt.rs:14-119).
#pragma once
#include <memory>
#include <vector>

#include "host_field.hpp"
#include "runtime.hpp"

namespace zkg {

struct CosetShift;

// The Groth16 quotient step fused into a forward transform's last pass: the transform's output
// c_i becomes (a_i b_i - c_i) zinv (a, b: plain Fr words, natural order; zinv a plain value).
struct Quotient {
  const uint32_t* a;
  const uint32_t* b;
  host::U256 zinv;
};

struct NttPlan {
  zkg_ctx* ctx;
  uint32_t log_n;
  std::vector<uint32_t> passes;  // stages per pass
  uint32_t n_inv_words[8];       // 1/n in Montgomery form
  // twiddles w^j, j < n/2: 8 words (R = 2^256) and five double limbs (R = 2^260) each
  DeviceArray scratch, fwd_tw, inv_tw, fwd_twd, inv_twd;
  // Seeds of the twiddle tables (two short tables of powers per direction), kept for the
  // plan's lifetime: freeing them would synchronise the whole device, which stalls a plan
  // made while other work runs (a server slot made under load).
  DeviceArray seeds[2][2];
  StageTimer timer;  // one stage id per pass

  NttPlan(zkg_ctx* ctx, uint32_t log_n);
  // Butterfly form: 0 = 32-bit integer products, 1 = double-precision limbs with twiddles read
  // from a table of w^j, 2 = double-precision limbs with each stage's twiddles staged into shared
  // memory from per-pass tables in butterfly order. Resets the pass split to the form's default.
  // The first switch to form 1 builds its twiddle limbs; form 2 builds its tables for each split
  // (set-up stream, waited for).
  bool set_variant(int variant);
  int variant = 2;
  uint32_t tile_log() const;
  // Splits the stages into passes of at most max_stages (6..tile_log()); false if not applicable
  // (transforms of one tile have a single pass).
  bool set_max_stages(uint32_t max_stages);
  uint32_t max_stages = 8;
  // Queues one transform of data (2^log_n elements) on stream s. With `shift` (inverse only),
  // the coset shift x_i <- x_i * g^i of that object is applied in the transform's last pass
  // (the same result as the transform followed by shift->enqueue, without another pass over
  // the data); the double-precision form runs the shift as its own kernel.
  // With `quot` (forward only), the output is (a b - NTT(data)) zinv instead (fused into the
  // last pass in forms 2 and 3; the other forms run the quotient kernel after the transform).
  void enqueue(uint32_t* data, bool inverse, cudaStream_t s, const CosetShift* shift = nullptr,
               const Quotient* quot = nullptr);
  void run(zkg_buf* data, bool inverse, const CosetShift* shift = nullptr, const Quotient* quot = nullptr);
  // Builds (on the set-up stream, then waits) the table a fused shift needs: the shift's
  // low powers times 1/n. enqueue makes it on first use; call this first when enqueue will be
  // captured into a graph.
  void prepare_shift(const CosetShift& shift);

 private:
  void build_seeds(const host::U256& root, DeviceArray (&seed)[2]);
  void build_twiddles(DeviceArray (&seed)[2], DeviceArray& out);
  // Form 2: one table per pass and direction, for the split in `passes`.
  void build_stage_tables();
  std::vector<std::unique_ptr<DeviceArray>> stage_tw[2];
  std::vector<uint32_t> stage_tw_mask;  // tables' block count - 1, per pass
  struct FusedShift {
    uint64_t serial;
    DeviceArray lo;  // n^-1 g^j, Montgomery form
  };
  std::vector<std::unique_ptr<FusedShift>> fused;
  const FusedShift* fused_for(const CosetShift& shift);
};

// x_i <- x_i * g^i over the first 2^log_n elements (plain Fr words), g fixed per object.
struct CosetShift {
  zkg_ctx* ctx;
  uint32_t log_n, lo_bits = 0;
  uint64_t serial;  // unique per object (keys the transforms' fused tables)
  DeviceArray hi, lo;  // powers g^(k * 2^lo_bits) and g^j, Montgomery form
  CosetShift(zkg_ctx* ctx, uint32_t log_n, const uint32_t* g_plain);
  void enqueue(uint32_t* data, cudaStream_t s);
  void run(zkg_buf* data);
};

// out_i <- (a_i * b_i - c_i) * zinv over 2^log_n plain Fr elements (zinv a plain value; out may
// be a or c).
void quotient(uint32_t* out, const uint32_t* a, const uint32_t* b, const uint32_t* c, uint32_t log_n,
              const host::U256& zinv, cudaStream_t s);
// (g^N - 1)^-1 for N = 2^log_n and a plain g < r: the inverse of the vanishing polynomial
// x^N - 1 anywhere on the coset g*H (ZKG_EINVAL when g^N = 1).
host::U256 coset_zinv(const uint32_t* g_plain, uint32_t log_n);

}  // namespace zkg

struct zkg_coset {
  zkg::CosetShift shift;
  zkg_coset(zkg_ctx* ctx, uint32_t log_n, const uint32_t* g) : shift(ctx, log_n, g) {}
};

struct zkg_ntt {
  zkg::NttPlan plan;
  zkg_ntt(zkg_ctx* ctx, uint32_t log_n) : plan(ctx, log_n) {}
};
