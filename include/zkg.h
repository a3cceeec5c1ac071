/* zkg.h — C ABI of the B200 (sm_100a) BN254 MSM and Fr NTT library.
 *
 * The entry points are exactly what a Rust (or any FFI) binding of zk-gpu's public API needs
 * (src/lib.rs:1-6 re-exports gpu, msm, ntt, group, host). Each declaration names the reference
 * interface it replaces as path:line within zerotruss/zk-gpu.
 *
 * Conventions
 *  - Plain pointers and sizes; opaque handles; no C++ or torch types.
 *  - Every fallible call returns ZKG_OK (0) or an error code; zkg_last_error() then returns a
 *    message for the calling thread. Argument errors carry the same text as the reference's
 *    panics (tests/invalid_inputs.rs:9-50), so a binding can panic with it unchanged.
 *  - Memory format (unchanged from the reference): 8 little-endian u32 words per field
 *    element; affine points are x then y, Fq2 coordinates a then b (x = a + b*u, u^2 = -1);
 *    the point at infinity is all-zero words (src/msm.rs:182-183, src/group.rs:59-69).
 *  - Work is queued on the context's single ordered stream and runs asynchronously until a
 *    read or zkg_ctx_sync, like the reference's wgpu queue (src/gpu.rs:151-155).
 *  - Results of the MSM are XYZZ points in Montgomery form with R = 2^256 (the reference's
 *    XYZZ words use R = 2^260; only the affine reading through zkg_xyzz_to_affine* is part of
 *    the contract, README.md:83-96).
 */
#ifndef ZKG_H
#define ZKG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct zkg_ctx zkg_ctx; /* gpu::Gpu                           src/gpu.rs:6-12   */
typedef struct zkg_buf zkg_buf; /* wgpu::Buffer of u32 words          src/gpu.rs:57-69  */
typedef struct zkg_msm zkg_msm; /* msm::Msm plan                      src/msm.rs:25-37  */
typedef struct zkg_ntt zkg_ntt; /* ntt::Ntt plan                      src/ntt.rs:14-20  */
typedef struct zkg_coset zkg_coset;
typedef struct zkg_batch zkg_batch; /* batched graph launch (no reference type, see below) */
typedef struct zkg_server zkg_server; /* proving-request server (no reference type, see below) */ /* coset shift by fixed g (no reference type, see below) */

enum zkg_status {
  ZKG_OK = 0,
  ZKG_EINVAL = 1,    /* argument out of range (the reference panics: msm.rs:97-98, ntt.rs:27) */
  ZKG_ESIZE = 2,     /* buffer too small (msm.rs:273-282, ntt.rs:53-59)                       */
  ZKG_ECUDA = 3,     /* CUDA runtime failure (wgpu device lost / validation, gpu.rs:44-49)     */
  ZKG_ENOMEM = 4,    /* device allocation failed                                               */
  ZKG_ETIMEDOUT = 5, /* a bounded device wait expired                                          */
  ZKG_ENODEV = 6     /* no usable GPU (Gpu::new_async's "no GPU adapter", gpu.rs:22-30)         */
};

enum zkg_group {
  ZKG_G1 = 1, /* group::Group::G1  src/group.rs:11-14 */
  ZKG_G2 = 2  /* group::Group::G2                     */
};

/* Message of the calling thread's last failed call ("" if none). */
const char *zkg_last_error(void);

/* ------------------------------------------------------------------ Gpu (src/gpu.rs) */

/* Gpu::new / Gpu::new_async (src/gpu.rs:22-55): context on CUDA device `device`. */
int zkg_ctx_new(int device, zkg_ctx **out);
void zkg_ctx_free(zkg_ctx *ctx);
/* Gpu::wait (src/gpu.rs:151-155): block until every queued call has finished; reports any
 * device fault that happened since the last check. */
int zkg_ctx_sync(zkg_ctx *ctx);
/* Gpu::adapter.name (src/gpu.rs:9): device name, NUL-terminated, truncated to cap. */
int zkg_ctx_device_name(zkg_ctx *ctx, char *out, size_t cap);

/* Gpu::buffer (src/gpu.rs:57-64): device buffer initialised with `words` u32 words. The host
 * array may be reused as soon as the call returns. */
int zkg_buf_new(zkg_ctx *ctx, const uint32_t *data, size_t words, zkg_buf **out);
/* Gpu::empty_buffer (src/gpu.rs:66-69): zero-filled buffer of `words` words. */
int zkg_buf_zeroed(zkg_ctx *ctx, size_t words, zkg_buf **out);
/* wgpu Queue::write_buffer: overwrite words [offset, offset + words) from host memory. */
int zkg_buf_write(zkg_ctx *ctx, zkg_buf *buf, size_t offset_words, const uint32_t *data, size_t words);
/* Gpu::read / try_read_async (src/gpu.rs:166-199): blocking copy of the first `words` words. */
int zkg_buf_read(zkg_ctx *ctx, const zkg_buf *buf, uint32_t *out, size_t words);

/* Asynchronous copies (no reference counterpart; wgpu's queue.write_buffer is itself queued).
 * zkg_buf_write_async queues a host-to-device copy on the context's upload stream: it starts
 * once the work already queued on the context that uses `buf` has finished (MSM runs, NTTs,
 * coset shifts, batch launches and asynchronous reads record their buffers), and work queued on
 * the context after the call waits for it. zkg_buf_read_async queues a device-to-host copy on
 * the read-back stream that runs after the last queued work that uses `buf` (every entry point
 * that queues work on a buffer records it); work queued after it that writes `buf` (an NTT or
 * coset shift of it, an MSM run of the plan whose result it is, a batch that holds it, a
 * write) waits for the copy, other work runs alongside it.
 * Neither call waits: `data` must stay unchanged, and `out` holds the words, only after
 * zkg_ctx_sync (which waits for both streams). From page-locked host memory (zkg_host_alloc)
 * the copies overlap the context's kernels. Size errors as zkg_buf_write / zkg_buf_read. */
int zkg_buf_write_async(zkg_ctx *ctx, zkg_buf *buf, size_t offset_words, const uint32_t *data, size_t words);
int zkg_buf_read_async(zkg_ctx *ctx, const zkg_buf *buf, uint32_t *out, size_t words);
/* wgpu Buffer::size / 4 */
size_t zkg_buf_words(const zkg_buf *buf);
/* Device address of the buffer, for interop with other CUDA code on the same device. */
void *zkg_buf_device_ptr(const zkg_buf *buf);
/* Frees a buffer made by zkg_buf_new / zkg_buf_zeroed / zkg_msm_upload_bases*. Borrowed
 * handles (zkg_msm_run's result) are ignored. */
void zkg_buf_free(zkg_buf *buf);

/* ------------------------------------------------------------------ Msm (src/msm.rs) */

/* Msm::default_window (src/msm.rs:76-80): clamp(log2(max(n,1)) - 5, 11, 16). */
uint32_t zkg_msm_default_window(size_t n);

/* Msm::upload_bases (src/msm.rs:182-188): affine points in plain coordinates (16 words per G1
 * point, 32 per G2 point; infinity (0,0)) converted on the device to Montgomery form. */
int zkg_msm_upload_bases(zkg_ctx *ctx, const uint32_t *plain_xy, size_t words, zkg_buf **out);
/* Msm::upload_bases_montgomery_256 (src/msm.rs:190-197): coordinates already in Montgomery
 * form with R = 2^256 (snarkjs / ffjavascript); with this library's R = 2^256 they are used
 * as they are. */
int zkg_msm_upload_bases_montgomery_256(zkg_ctx *ctx, const uint32_t *xy, size_t words, zkg_buf **out);

/* Msm::for_group / new / with_item_points (src/msm.rs:82-180). `c` must be in 9..=20;
 * item_points = 0 picks the work-item size automatically (points accumulated per thread
 * before partial sums are combined). Fails with the reference's messages: "an MSM needs at
 * least one point", "window size c must be in 9..=20, got {c}". */
int zkg_msm_new(zkg_ctx *ctx, int group, size_t n, uint32_t c, uint32_t item_points, zkg_msm **out);
void zkg_msm_free(zkg_msm *msm);
/* Msm::group (src/msm.rs:267-269) */
int zkg_msm_group(const zkg_msm *msm);
/* Tuning knobs of a plan (no reference counterpart): the accumulation kernel's form, 0 = field
 * products inlined, 1 = products through one out-of-line function (smaller code),
 * 2 = out of line, two independent products per call, 3 / 4 = bucket sums in double-precision
 * limbs, products on the FP64 pipe, two per call / one per call (bit-exact for G1 and G2; the
 * G2 limb forms are slower than the integer pairs). Defaults: for G1 4 (with the plain windows, 3
 * below 2^26 (window, point) entries and 4 from there), for G2 2.
 * zkg_msm_params reports the plan's window c, points per accumulation thread and form. */
int zkg_msm_set_variant(zkg_msm *msm, int variant);
/* Counting-sort knob (no reference counterpart): how a warp merges the counting pass's atomics
 * for lanes whose digits hit the same (window, bucket) slot: 0 = every group of equal slots,
 * 1 = the group of the first lane only, 2 = none, 3 = the group of the first pair of
 * neighbouring lanes with equal slots (default). The scatter pass always merges every group. */
int zkg_msm_set_sort(zkg_msm *msm, int mode);
/* Counting-sort form (no reference counterpart): 0 = one pass scatters every (window, point)
 * entry through an atomic cursor per slot; 1 = the counting pass also records each entry's
 * rank within its slot (and its digit), and the placing pass writes the entries window by
 * window, so the stores of one window meet in L2 (default; applies for c <= 16, larger c use 0;
 * 6 more bytes of plan memory per (window, point) entry). */
int zkg_msm_set_sort_form(zkg_msm *msm, int form);
/* Fixed-base MSM over a resident key (no reference counterpart: the reference combines its
 * windows by Horner, msm_combine.wgsl:13-22, on every run). zkg_msm_fixed_base_table builds, once
 * per key and window size c, a table of ceil(255/c) rows of n points, row w holding 2^(c w) P_i
 * (affine, Montgomery form, infinity as zeros; the bases as zkg_msm_upload_bases* made them).
 * A plan with zkg_msm_set_fixed_base(msm, 1) then takes that table as its `bases`: the digits of
 * every window go to one set of 2^(c-1) buckets (point w * n + i of the table), so a run has one
 * bucket reduction instead of one per window and no doublings between windows; the result is
 * the same point as the plain MSM over the key. Needs c <= 16 and windows * n < 2^31; the
 * table holds windows times the key's memory. */
int zkg_msm_fixed_base_table(zkg_ctx *ctx, int group, const zkg_buf *bases, size_t n, uint32_t c, zkg_buf **out);
int zkg_msm_set_fixed_base(zkg_msm *msm, int enable);
/* GLV splitting for G1 (no reference counterpart; the reference names GLV as a next step,
 * README.md:223-224): with enable = 1 every scalar k is split as k1 + k2 lambda (mod r), |k1|,
 * |k2| < 2^127, and a run sums k1_i P_i + k2_i phi(P_i) with phi(x, y) = (beta x, y): 2n points
 * (the plan makes phi(P_i) from `bases` on every run, 64 more bytes of plan memory per point)
 * with W = ceil(128 / c) windows instead of ceil(255 / c), the 128 bits spread over them as
 * evenly as possible (widths floor(128 / W) or one more, never above c), so about the same number
 * of bucket additions and half the bucket reductions and combination doublings. The result is the same point as the
 * plain MSM (scalars are taken mod r). On by default for G1 plans with c <= 16 and n < 2^30
 * (measured faster at every default window); enable = 1 elsewhere (G2, c > 16, a fixed-base
 * plan) is ZKG_EINVAL; zkg_msm_set_fixed_base(msm, 1) switches it off. Re-sizes the plan's
 * scratch (synchronises with queued work). zkg_msm_windows reports the plan's window count and
 * whether GLV is on. */
int zkg_msm_set_glv(zkg_msm *msm, int enable);
int zkg_msm_windows(const zkg_msm *msm, uint32_t *windows, int *glv);
/* Runs in passes (no reference counterpart; the reference sizes one pass for n < 2^31,
 * src/shaders/msm_digits.wgsl:33). Entry positions and point indices are 32-bit, so one pass holds
 * fewer than 2^32 (window, point) entries (about 2^28 points at c = 16); a plan over more points
 * runs over consecutive slices of at most `chunk` points and adds their results, so every n <
 * 2^31 works. The plan's scratch is sized for one slice: zkg_msm_set_chunk(msm, points) sets a
 * smaller slice to bound the plan's device memory (0 restores the largest; values above it are
 * clamped; re-sizes the scratch, synchronising with queued work). A fixed-base plan runs in one
 * pass (ZKG_EINVAL). zkg_msm_passes reports the slice and the number of passes. The result is
 * the same point for every slice size. */
int zkg_msm_set_chunk(zkg_msm *msm, size_t points);
int zkg_msm_passes(const zkg_msm *msm, size_t *chunk, size_t *passes);
int zkg_msm_params(const zkg_msm *msm, uint32_t *c, uint32_t *item_points, int *variant);
/* Msm::run (src/msm.rs:284-298): queue sum(scalars[i] * bases[i]); scalars are 8 plain u32
 * words each. *result is a borrowed handle to the plan's XYZZ result (32 words G1, 64 words G2,
 * Montgomery form), overwritten by the next run. Checks sizes first ("scalars buffer holds ...",
 * "bases buffer holds ..."). */
int zkg_msm_run(zkg_msm *msm, const zkg_buf *bases, const zkg_buf *scalars, const zkg_buf **result);

typedef struct {
  char stage[32];
  double ms;
} zkg_stage_time;
/* Msm::profile (src/msm.rs:321-342): runs every stage separately and reports device time per
 * stage (CUDA events). *count receives the number of stages written (at most cap). */
int zkg_msm_profile(zkg_msm *msm, const zkg_buf *bases, const zkg_buf *scalars, zkg_stage_time *out, size_t cap,
                    size_t *count);

/* xyzz_to_affine (src/msm.rs:345-354): 32 result words -> plain affine x, y as 4 LE u64 each.
 * Returns 1 for a finite point, 0 for infinity (x, y set to zero), negative on error. */
int zkg_xyzz_to_affine(const uint32_t *words, uint64_t *x, uint64_t *y);
/* xyzz_to_affine_g2 (src/msm.rs:356-373): 64 words -> x = (x.a, x.b), y = (y.a, y.b), each
 * coordinate 4 LE u64 (8 u64 per Fq2 value). Returns 1 finite, 0 infinity. */
int zkg_xyzz_to_affine_g2(const uint32_t *words, uint64_t *x, uint64_t *y);
/* P + Q for two XYZZ points in this library's memory format (32 words G1, 64 G2; R = 2^256
 * Montgomery words; infinity has ZZ = 0), on the host: combines the partial results of MSMs
 * that several GPUs ran over shards of one key (no reference counterpart: the reference runs on
 * one device). add-2008-s / dbl-2008-s-1 with every special case; out may alias a or b. */
int zkg_xyzz_add_host(int group, const uint32_t *a, const uint32_t *b, uint32_t *out);

/* ------------------------------------------------------------------ Ntt (src/ntt.rs) */

/* Ntt::new (src/ntt.rs:26-40): plan for 2^log_n elements, 10 <= log_n <= 27
 * ("log_n must be in 10..=27"). */
int zkg_ntt_new(zkg_ctx *ctx, uint32_t log_n, zkg_ntt **out);
void zkg_ntt_free(zkg_ntt *ntt);
/* Ntt::log_n (src/ntt.rs:19) */
uint32_t zkg_ntt_log_n(const zkg_ntt *ntt);
/* Ntt::forward (src/ntt.rs:42-45): in place, natural order in and out (plain Fr words).
 * Fails with "data buffer holds ..." if the buffer is smaller than 2^log_n elements. */
int zkg_ntt_forward(zkg_ntt *ntt, zkg_buf *data);
/* Ntt::inverse (src/ntt.rs:47-50): in place, includes the 1/n factor. */
int zkg_ntt_inverse(zkg_ntt *ntt, zkg_buf *data);

/* Coset shift x_i <- x_i * g^i over the first 2^log_n plain Fr elements of a buffer, for a
 * fixed g < r given as 8 plain words: the distribute-powers step of a Groth16 witness map
 * between an inverse and a forward transform. The reference leaves it to callers ("coset
 * shifts ... are simple kernels on top", README.md:229-230); there is no reference function.
 * zkg_coset_new precomputes two small power tables (about 2^(log_n/2) elements each). */
int zkg_coset_new(zkg_ctx *ctx, uint32_t log_n, const uint32_t *g, zkg_coset **out);
void zkg_coset_free(zkg_coset *coset);
int zkg_coset_shift(zkg_coset *coset, zkg_buf *data);
/* zkg_ntt_inverse then zkg_coset_shift in one call, the shift applied in the inverse's last pass
 * (its 1/n factor folded into the shift's table): the same words as the two calls, one pass
 * over the data fewer. The coset must cover 2^log_n elements of the transform. */
int zkg_ntt_inverse_coset(zkg_ntt *ntt, zkg_buf *data, zkg_coset *coset);

/* The pointwise step of a Groth16 witness map on the coset g*H, H the 2^log_n-th roots of unity
 * (the reference leaves it to callers: "coset shifts and pointwise products, which are simple
 * kernels on top", README.md:229-230; no reference function): with a, b, c the evaluations of
 * the three constraint polynomials on g*H, h_i = (a_i b_i - c_i) / (g^N - 1), N = 2^log_n (the
 * vanishing polynomial x^N - 1 takes the value g^N - 1 everywhere on the coset). All plain Fr
 * words, natural order; g < r given as 8 plain words, g^N != 1 (ZKG_EINVAL otherwise). */
/* a <- h. */
int zkg_quotient(zkg_ctx *ctx, zkg_buf *a, const zkg_buf *b, const zkg_buf *c, uint32_t log_n, const uint32_t *g);
/* zkg_ntt_forward of data (c's coefficients, already shifted onto the coset), then
 * data <- (a b - data) / (g^N - 1) with N the transform's size: the quotient runs in the
 * transform's last pass (forms 2 and 3), saving a kernel and a read and a write of c; the same
 * words as zkg_ntt_forward followed by zkg_quotient into c. */
int zkg_ntt_forward_quotient(zkg_ntt *ntt, zkg_buf *data, const zkg_buf *a, const zkg_buf *b, const uint32_t *g);

/* ------------------------------------------------------------------ proving keys (.zkey)
 * The on-disk form behind zkg_msm_upload_bases_montgomery_256 (Msm::upload_bases_montgomery_256,
 * src/msm.rs:190-197, documented there as "the form ffjavascript and snarkjs keep points in";
 * the reference has no reader: its callers parse the file, README.md:104-105). A snarkjs
 * Groth16 .zkey over BN254 is parsed on the host (no GPU needed); its point sections are then
 * uploaded as resident MSM bases without conversion. Sections: */
#define ZKG_ZKEY_IC 3 /* nPublic + 1 G1 points */
#define ZKG_ZKEY_A 5  /* nVars G1 */
#define ZKG_ZKEY_B1 6 /* nVars G1 */
#define ZKG_ZKEY_B2 7 /* nVars G2 */
#define ZKG_ZKEY_C 8  /* nVars - nPublic - 1 G1 */
#define ZKG_ZKEY_H 9  /* domainSize G1 */
typedef struct zkg_zkey zkg_zkey;
typedef struct {
  uint32_t protocol; /* 1 = Groth16 */
  uint32_t n_vars, n_public, domain_size;
} zkg_zkey_header;
/* Parses a file image (bytes stay the caller's; the key keeps its own copy of the points).
 * ZKG_EINVAL with the reason for a malformed file, another protocol, another curve, a section
 * whose size does not match the header, or a coordinate not below q. */
int zkg_zkey_parse(const void *bytes, size_t len, zkg_zkey **out);
void zkg_zkey_free(zkg_zkey *zkey);
int zkg_zkey_info(const zkg_zkey *zkey, zkg_zkey_header *out);
/* A point section as the file holds it: 16 (G1) or 32 (G2) words per point, Montgomery form
 * with R = 2^256, infinity as zeros; *words stays valid until zkg_zkey_free. */
int zkg_zkey_points(const zkg_zkey *zkey, uint32_t section, const uint32_t **words, size_t *points, int *group);
/* zkg_msm_upload_bases_montgomery_256 of a point section: resident bases for zkg_msm_run. */
int zkg_zkey_upload(zkg_ctx *ctx, const zkg_zkey *zkey, uint32_t section, zkg_buf **out);

/* ------------------------------------------------------------------ autotuning
 * No reference counterpart (its parameters are fixed: default_window, item size, TILE_LOG).
 * zkg_tune_msm times, on the given inputs, windows c in [default_window(n) - 2, + 2] within
 * 9..=20, 16..256 points per accumulation thread, the accumulation kernel forms and, for G1 with
 * c <= 16, the GLV split on and off, and writes
 * up to cap results fastest first (out[0] is the choice; *count receives how many).
 * zkg_ntt_set_variant picks a plan's butterfly form: 0 = 32-bit integer products (tiles of 2^11
 * elements; default), 1 = double-precision limbs, products on the FP64 pipe (tiles of 2^10);
 * it resets the pass split to the form's default (at most 9 / 8 stages per pass).
 * zkg_ntt_set_max_stages picks the pass split (at most max_stages, 6..=11 for form 0, 6..=10
 * for form 1, stages per shared-memory pass); zkg_ntt_params reports form, split and passes.
 * zkg_tune_ntt times both forms and each split on `data` (forward + inverse, which leaves the
 * data unchanged) and returns the best. */
typedef struct {
  uint32_t c, item_points;
  int variant;
  int glv; /* zkg_msm_set_glv */
  double ms;
} zkg_msm_tuning;
int zkg_tune_msm(zkg_ctx *ctx, int group, size_t n, const zkg_buf *bases, const zkg_buf *scalars, int reps,
                 zkg_msm_tuning *out, size_t cap, size_t *count);
int zkg_ntt_set_variant(zkg_ntt *ntt, int variant);
int zkg_ntt_set_max_stages(zkg_ntt *ntt, uint32_t max_stages);
int zkg_ntt_params(const zkg_ntt *ntt, int *variant, uint32_t *max_stages, uint32_t *passes);
int zkg_tune_ntt(zkg_ctx *ctx, uint32_t log_n, zkg_buf *data, int reps, int *best_variant, uint32_t *best_max_stages,
                 double *best_ms);

/* ------------------------------------------------------------------ batched execution
 * No reference counterpart: the reference submits one command buffer per stage per call
 * (src/msm.rs:286-298, src/ntt.rs:52-68). A batch records MSMs, NTTs and coset shifts on
 * lanes (0 <= lane < 64) and captures them into one CUDA graph: operations in a lane run in
 * order, lanes are independent branches that the device overlaps. One plan may be used in one
 * lane only (its scratch is its own). zkg_batch_launch replays the graph on the context stream
 * with a single launch (capturing first if operations were added since the last capture).
 * Buffers and plans must stay alive while the batch exists. MSM results are copied into
 * `result` (>= 32 words G1, 64 words G2), so a plan may run several times in its lane. */
int zkg_batch_new(zkg_ctx *ctx, zkg_batch **out);
void zkg_batch_free(zkg_batch *batch);
int zkg_batch_add_msm(zkg_batch *batch, zkg_msm *msm, const zkg_buf *bases, const zkg_buf *scalars, zkg_buf *result,
                      int lane);
int zkg_batch_add_ntt(zkg_batch *batch, zkg_ntt *ntt, zkg_buf *data, int inverse, int lane);
int zkg_batch_add_coset(zkg_batch *batch, zkg_coset *coset, zkg_buf *data, int lane);
int zkg_batch_capture(zkg_batch *batch);
int zkg_batch_launch(zkg_batch *batch);
/* The same operations without a graph: one stream per lane, joined into the context stream. */
int zkg_batch_run_streams(zkg_batch *batch);
/* Kernel nodes in the captured graph (0 before the first capture). */
size_t zkg_batch_kernels(const zkg_batch *batch);

/* ------------------------------------------------------------------ serving
 * No reference counterpart (its callers issue one call at a time). A server keeps proving keys
 * resident and runs Groth16-shaped requests: three G1 MSMs (sizes g1_count[0..2] <= m) and one
 * G2 MSM (m) over the smallest resident key with at least m = 2^log_m points, and a witness-map
 * chain of seven Fr NTTs of size N = 2m on the evaluation vectors a, b, c:
 *   p <- forward(shift_g(inverse(p))) for p in a, b, c;  h <- (a*b - c) / (g^N - 1);
 *   h <- shift_{1/g}(inverse(h)).
 * Outputs: out_points = 3 G1 XYZZ (32 words each) then 1 G2 XYZZ (64 words); out_h = N elements.
 * Requests queue FIFO; while fewer than `lanes` run, the queue is scanned in order: a request
 * with an idle slot (plans and buffers of its size) starts at once, one without has a slot made
 * for it on a builder thread when that fits the HBM budget (idle slots of other sizes are
 * evicted), and the scan goes on past it; a request whose slot does not fit holds back the ones
 * behind it. Up to `lanes` requests run at once on separate streams, each as one captured CUDA
 * graph with three parallel branches (continuous batching). plain = 1 is the one-call-at-a-time path: one request at a
 * time, operations launched one by one. Host buffers of a request must stay valid until
 * zkg_server_wait returns for it, and should be page-locked (zkg_host_alloc) for overlap. */
typedef struct {
  int lanes;               /* requests on the device at once, 1..64 (plain forces 1) */
  int plain;               /* 1 = one request at a time, no graphs, no branches */
  size_t hbm_budget_bytes; /* device memory for slots; 0 = 80% of the free memory at creation */
  uint32_t coset_g[8];     /* coset generator g, plain Fr words, 0 < g < r */
} zkg_server_config;
typedef struct {
  uint32_t log_m;                 /* 11..26 */
  const uint32_t *g1_scalars[3];  /* g1_count[j] scalars each, 8 words per scalar */
  size_t g1_count[3];
  const uint32_t *g2_scalars;     /* m scalars */
  const uint32_t *polys[3];       /* a, b, c: N = 2m plain Fr elements each */
  uint32_t *out_points;           /* 3*32 + 64 words */
  uint32_t *out_h;                /* N elements (8*N words) */
} zkg_proof_request;
typedef struct {
  double queued_ms, device_ms, total_ms;  /* submit -> admitted -> done */
} zkg_request_times;
typedef struct {
  uint64_t queued, completed, slots, slots_created, slots_evicted;
  size_t bytes_used, budget;
  double build_ms; /* host time spent making slots */
} zkg_server_counters;
int zkg_server_new(zkg_ctx *ctx, const zkg_server_config *config, zkg_server **out);
/* Waits for every queued request, then frees the server (keys' buffers stay the caller's). */
void zkg_server_free(zkg_server *server);
/* A resident proving key: n affine points in G1 and in G2, Montgomery form (as made by
 * zkg_msm_upload_bases*). The buffers must outlive the server. */
int zkg_server_add_key(zkg_server *server, size_t n, const zkg_buf *g1_bases, const zkg_buf *g2_bases);
int zkg_server_submit(zkg_server *server, const zkg_proof_request *request, uint64_t *id);
/* Blocks until the request is done (timeout_ms < 0: no limit; ZKG_ETIMEDOUT otherwise). */
int zkg_server_wait(zkg_server *server, uint64_t id, int timeout_ms, zkg_request_times *times);
int zkg_server_stats(zkg_server *server, zkg_server_counters *stats);
/* Makes idle slots of size 2^log_m until the server holds `count` of them (a warm server: a
 * burst of requests of that size does not wait for slot construction). ZKG_ENOMEM when a slot
 * does not fit the HBM budget. */
int zkg_server_reserve(zkg_server *server, uint32_t log_m, uint32_t count);

/* Largest transform zkg_ntt_noalloc accepts: 2^16 elements. */
#define ZKG_NTT_NOALLOC_MAX_LOG_N 16
/* No counterpart in the reference (its Ntt always owns a scratch buffer, src/ntt.rs:31).
 * In-place Fr NTT of 2^log_n elements (10 <= log_n <= ZKG_NTT_NOALLOC_MAX_LOG_N) in the
 * caller's device buffer `data` (8 plain words per element, 16-byte aligned), natural order
 * in and out, the inverse with the 1/n factor; bit-identical to zkg_ntt_forward/inverse.
 * It allocates no device memory, for callers that cannot call cudaMalloc (a device-memory
 * budget owned by another allocator, a pipeline where allocation is not allowed): its scratch
 * is one static device array of 3 MiB that every GPU which loads this library holds until the
 * process exits. Work is queued on `stream` (a cudaStream_t; NULL = the legacy default stream)
 * of the calling thread's current device. The first call on a device also resolves the array's
 * address for that device (cudaGetSymbolAddress) and sets the kernels' shared-memory limit;
 * make that first call before any stream capture. After cudaDeviceReset the device has a new
 * context, and the next call resolves the address again (again: not during a capture). All calls share the array, which keeps the
 * last call's contents: calls that overlap on the GPU (different streams, or different host
 * threads on one device) race and give wrong results; order them on one stream. Larger sizes
 * are rejected with ZKG_EINVAL ("log_n must be in 10..=16 for zkg_ntt_noalloc, got N"). */
int zkg_ntt_noalloc(uint32_t log_n, int inverse, uint32_t *data, void *stream);

/* ------------------------------------------------------------------ runtime helpers (no reference counterpart:
 * wgpu hides its queue, launches and staging memory) */

/* The context's cudaStream_t, for callers that time or order work with their own CUDA calls. */
void *zkg_ctx_stream(zkg_ctx *ctx);
/* Number of kernels this library has launched in this process (all contexts). */
uint64_t zkg_launch_count(void);
/* Page-locked host memory for fast host<->device copies (cudaHostAlloc / cudaFreeHost). */
int zkg_host_alloc(size_t bytes, void **out);
void zkg_host_free(void *p);

/* Live stage timing: while enabled, every zkg_msm_run records CUDA events around each stage on
 * the context stream (no synchronisation); zkg_msm_stage_times waits for them, returns the
 * summed device time per stage over the runs since the last call, and starts a new sum.
 * *runs receives the number of runs summed. */
int zkg_msm_set_timing(zkg_msm *msm, int enable);
int zkg_msm_stage_times(zkg_msm *msm, zkg_stage_time *out, size_t cap, size_t *count, size_t *runs);
/* Number of (point, window) entries with a nonzero digit in the last run (blocking): the
 * mixed additions the accumulation performed, for throughput accounting (for a plan that runs
 * in passes, zkg_msm_passes, those of the last pass). */
int zkg_msm_last_entries(zkg_msm *msm, uint64_t *entries);
/* The same for the NTT: one entry per pass ("pass 0", "pass 1", ...), forward and inverse
 * transforms summed together. */
int zkg_ntt_set_timing(zkg_ntt *ntt, int enable);
int zkg_ntt_pass_times(zkg_ntt *ntt, zkg_stage_time *out, size_t cap, size_t *count, size_t *runs);

/* ------------------------------------------------------------------ testing and set-up helpers */

/* Peak-rate probes, the denominators of the measured roofline fractions (the reference's
 * examples/field_bench.rs measures mulmods per second the same way): variant 0 = mad.lo.u32,
 * 1 = mad.hi.u32, 2 = carry-chained mad.lo.cc / madc.hi.cc (the Montgomery rows' form), 3 = Fq
 * Montgomery products (integer form), 9 = fma.rn.f64 (the double-precision pipe), 11 = Fq
 * Montgomery products on the double-precision pipe (five 52-bit limbs, R = 2^260; checked on the
 * device against the integer form before it is timed). Other variants: ZKG_EINVAL.
 * *ops_per_second receives multiply-adds (or products, or FMAs) per second on the context's
 * device; the best of five launches over every SM. */
int zkg_bench_integer_pipe(zkg_ctx *ctx, int variant, double *ops_per_second);

/* Point operations for the curve tests (the reference's tests/curve.rs:22-44 kernel): for each
 * of `count` affine pairs (P, Q) in Montgomery form (32 words G1 / 64 words G2 per pair), writes
 * three XYZZ points: P + Q (mixed add), 2P (double), (P + Q) + 2P (full add). */
int zkg_test_point_ops(zkg_ctx *ctx, int group, const uint32_t *pairs, size_t count, uint32_t *out);

/* The device's GLV split (zkg_msm_set_glv) of `count` scalars in host memory (8 words each):
 * out[10 i ..] = |k1| (4 words), |k2| (4 words), sign of k1, sign of k2 (1 = negative), with k =
 * k1 + k2 lambda (mod r), lambda = 0x30644e72e131a029048b6e193fd84104cc37a73fec2bc5e9b8ca0b2d36636f23. */
int zkg_test_glv_split(zkg_ctx *ctx, const uint32_t *scalars, size_t count, uint32_t *out);

/* Fixed-base batch multiplication: out[i] = [k_i] G for the standard generator of `group`
 * (G1 = (1, 2)), as affine points in plain (mont256 = 0) or Montgomery-2^256 (mont256 = 1)
 * coordinates. Scalars are 8 words each, any 256-bit value. Used to build proving-key-like
 * bases on the device (the reference's tests build them with arkworks, tests/g2.rs:136). */
int zkg_generator_multiples(zkg_ctx *ctx, int group, const zkg_buf *scalars, size_t n, int mont256, zkg_buf *out);

#ifdef __cplusplus
}
#endif

#endif /* ZKG_H */
