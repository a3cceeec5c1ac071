/* C restatement of zk-gpu's BN254 MSM and Fr NTT: the oracle for large inputs and the
 * timed multi-threaded CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY. Loaded (through ctypes) by the tests, by the smoke check and
 * by the CPU-baseline leg of bench.py, and never by the product library.
 *
 * What it restates, with the reference location it follows:
 *   signed c-bit digits with carry, W = ceil(255/c) .... src/shaders/msm_digits.wgsl:19-37,
 *                                                        src/msm.rs:101
 *   bucket accumulation (XYZZ mixed adds) .............. src/shaders/msm_accumulate.wgsl:38-44
 *   running-sum bucket reduction sum_b (b+1)*B_b ....... src/shaders/msm_reduce_chunks.wgsl:26-40
 *   Horner window combination .......................... src/shaders/msm_combine.wgsl:13-22
 *   Msm::upload_bases / upload_bases_montgomery_256 .... src/msm.rs:182-197
 *   NTT: root 5^((r-1)>>log_n), DIF radix-2, natural
 *   order in/out, inverse with the 1/n factor .......... src/ntt.rs:26-68, src/host.rs:94-98,
 *                                                        src/shaders/ntt.wgsl:50-73
 * The multi-threaded structure (windows x point chunks for the MSM, stage-parallel then
 * block-local passes for the NTT) stands in for arkworks' rayon-parallel VariableBaseMSM and
 * Radix2EvaluationDomain::fft (examples/bench.rs:160-164,216-218), which cannot be built here.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_field.h"

/* ---------------------------------------------------------------- curve instantiations */
#define P_ g1_
#define T_ fe
#define ADD_ fq_add_
#define SUB_ fq_sub_
#define MUL_ fq_mul_
#define NEG_ fq_neg_
#define INV_ fq_inv_
#define IS_ZERO_ fe_is_zero
#define ONE_ FQ_F.one
#include "oracle_curve.h"
#undef P_
#undef T_
#undef ADD_
#undef SUB_
#undef MUL_
#undef NEG_
#undef INV_
#undef IS_ZERO_
#undef ONE_

static const fe2 FQ2_ONE = {{{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}},
                            {{0, 0, 0, 0}}};
#define P_ g2_
#define T_ fe2
#define ADD_ fe2_add
#define SUB_ fe2_sub
#define MUL_ fe2_mul
#define NEG_ fe2_neg
#define INV_ fe2_inv
#define IS_ZERO_ fe2_is_zero
#define ONE_ FQ2_ONE
#include "oracle_curve.h"
#undef P_
#undef T_
#undef ADD_
#undef SUB_
#undef MUL_
#undef NEG_
#undef INV_
#undef IS_ZERO_
#undef ONE_

/* ---------------------------------------------------------------- threads */
typedef void (*task_fn)(void *ctx, int tid, int nthreads);
typedef struct { task_fn fn; void *ctx; int tid, n; } thread_arg;

static void *thread_main(void *p) {
  thread_arg *a = (thread_arg *)p;
  a->fn(a->ctx, a->tid, a->n);
  return NULL;
}

static void run_parallel(int nthreads, task_fn fn, void *ctx) {
  if (nthreads <= 1) { fn(ctx, 0, 1); return; }
  pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
  thread_arg *args = (thread_arg *)malloc(sizeof(thread_arg) * nthreads);
  for (int t = 0; t < nthreads; t++) {
    args[t].fn = fn; args[t].ctx = ctx; args[t].tid = t; args[t].n = nthreads;
    if (t > 0) pthread_create(&th[t], NULL, thread_main, &args[t]);
  }
  fn(ctx, 0, nthreads);
  for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
  free(th);
  free(args);
}

/* ---------------------------------------------------------------- signed digits */
static inline uint32_t window_bits(const uint32_t *s, int pos, int c) {
  int word = pos >> 5, off = pos & 31;
  uint64_t v = 0;
  if (word < 8) v = s[word] >> off;
  if (off + c > 32 && word + 1 < 8) v |= (uint64_t)s[word + 1] << (32 - off);
  return (uint32_t)(v & ((1u << c) - 1));
}

typedef struct {
  const uint32_t *scalars;
  size_t n;
  int c, windows;
  int32_t *digits; /* [windows][n] */
} digits_ctx;

static void digits_task(void *p, int tid, int nt) {
  digits_ctx *d = (digits_ctx *)p;
  size_t lo = d->n * tid / nt, hi = d->n * (tid + 1) / nt;
  uint32_t half = 1u << (d->c - 1);
  for (size_t i = lo; i < hi; i++) {
    uint32_t carry = 0;
    for (int w = 0; w < d->windows; w++) {
      uint32_t v = window_bits(d->scalars + 8 * i, w * d->c, d->c) + carry;
      int32_t digit = (int32_t)v;
      carry = 0;
      if (v >= half) { digit = (int32_t)v - (1 << d->c); carry = 1; }
      d->digits[(size_t)w * d->n + i] = digit;
    }
  }
}

/* ---------------------------------------------------------------- MSM (both groups) */
typedef struct {
  int group;
  const void *bases;   /* g1_aff[] or g2_aff[] in Montgomery form */
  size_t n;
  int c, windows, chunks;
  const int32_t *digits;
  void *partials;      /* [windows][chunks] xyzz */
  int next_task;
  pthread_mutex_t lock;
} msm_ctx;

#define MSM_TASK_BODY(G)                                                                      \
  do {                                                                                        \
    G##xyzz *buckets = (G##xyzz *)malloc(sizeof(G##xyzz) * half);                             \
    const G##aff *bases = (const G##aff *)m->bases;                                           \
    for (;;) {                                                                                \
      pthread_mutex_lock(&m->lock);                                                           \
      int task = m->next_task++;                                                              \
      pthread_mutex_unlock(&m->lock);                                                         \
      if (task >= m->windows * m->chunks) break;                                              \
      int w = task / m->chunks, k = task % m->chunks;                                         \
      size_t lo = m->n * k / m->chunks, hi = m->n * (k + 1) / m->chunks;                      \
      memset(buckets, 0, sizeof(G##xyzz) * half);                                             \
      const int32_t *dg = m->digits + (size_t)w * m->n;                                       \
      for (size_t i = lo; i < hi; i++) {                                                      \
        int32_t d = dg[i];                                                                    \
        if (d == 0) continue;                                                                 \
        if (d > 0) {                                                                          \
          G##add_aff(&buckets[d - 1], &buckets[d - 1], &bases[i]);                            \
        } else {                                                                              \
          G##aff neg;                                                                         \
          G##aff_neg(&neg, &bases[i]);                                                        \
          G##add_aff(&buckets[-d - 1], &buckets[-d - 1], &neg);                               \
        }                                                                                     \
      }                                                                                       \
      G##xyzz run, tot;                                                                       \
      G##set_inf(&run);                                                                       \
      G##set_inf(&tot);                                                                       \
      for (int64_t b = (int64_t)half - 1; b >= 0; b--) {                                      \
        G##add(&run, &run, &buckets[b]);                                                      \
        G##add(&tot, &tot, &run);                                                             \
      }                                                                                       \
      ((G##xyzz *)m->partials)[(size_t)w * m->chunks + k] = tot;                              \
    }                                                                                         \
    free(buckets);                                                                            \
  } while (0)

static void msm_task(void *p, int tid, int nt) {
  (void)tid; (void)nt;
  msm_ctx *m = (msm_ctx *)p;
  size_t half = (size_t)1 << (m->c - 1);
  if (m->group == 1) MSM_TASK_BODY(g1_); else MSM_TASK_BODY(g2_);
}

/* Window size like arkworks' VariableBaseMSM: ln(n) + 2 (ln ~ 0.69 log2). */
static int cpu_window(size_t n) {
  if (n < 32) return 3;
  int lg = 0;
  while (((size_t)1 << (lg + 1)) <= n) lg++;
  int c = lg * 69 / 100 + 2;
  return c < 2 ? 2 : (c > 20 ? 20 : c);
}

/* Loads n affine points (plain, or Montgomery-2^256 if mont256) into Montgomery form. */
static void *load_bases(int group, const uint32_t *w, int mont256, size_t n) {
  size_t coords = n * (group == 1 ? 2 : 4);
  fe *out = (fe *)malloc(sizeof(fe) * coords);
  for (size_t i = 0; i < coords; i++) {
    fe_from_words(&out[i], w + 8 * i);
    if (!mont256) fe_to_mont(&out[i], &out[i], &FQ_F);
  }
  return out;
}

/* sum_i scalars[i] * bases[i]. bases: 16 (G1) or 32 (G2) words per point, plain or
 * Montgomery-2^256 coordinates, infinity = all zero; scalars: 8 words each.
 * out: plain affine words (zeros = infinity). c = 0 picks the CPU window. */
int oracle_msm(int group, const uint32_t *bases_words, int mont256, const uint32_t *scalars, size_t n,
               int c, int threads, uint32_t *out) {
  if (group != 1 && group != 2) return -1;
  size_t aw = group == 1 ? 16 : 32;
  memset(out, 0, aw * 4);
  if (n == 0) return 0;
  if (c <= 0) c = cpu_window(n);
  if (c < 2 || c > 22) return -2;
  if (threads < 1) threads = 1;
  int windows = (255 + c - 1) / c;
  digits_ctx d = {scalars, n, c, windows, (int32_t *)malloc(sizeof(int32_t) * n * windows)};
  run_parallel(threads, digits_task, &d);

  msm_ctx m;
  m.group = group;
  m.bases = load_bases(group, bases_words, mont256, n);
  m.n = n; m.c = c; m.windows = windows;
  size_t half = (size_t)1 << (c - 1);
  /* Enough tasks to keep every thread busy, while each chunk stays large next to the
   * 2 * half bucket-reduction additions it pays for. */
  int chunks = (2 * threads + windows - 1) / windows;
  while (chunks > 1 && n / chunks < 4 * half) chunks--;
  m.chunks = chunks;
  m.digits = d.digits;
  m.next_task = 0;
  pthread_mutex_init(&m.lock, NULL);
  size_t xs = group == 1 ? sizeof(g1_xyzz) : sizeof(g2_xyzz);
  m.partials = malloc(xs * windows * chunks);
  run_parallel(threads, msm_task, &m);
  pthread_mutex_destroy(&m.lock);

  if (group == 1) {
    g1_xyzz *ps = (g1_xyzz *)m.partials, acc, sw;
    g1_set_inf(&acc);
    for (int w = windows - 1; w >= 0; w--) {
      for (int k = 0; k < c && w < windows - 1; k++) g1_dbl(&acc, &acc);
      g1_set_inf(&sw);
      for (int k = 0; k < chunks; k++) g1_add(&sw, &sw, &ps[(size_t)w * chunks + k]);
      g1_add(&acc, &acc, &sw);
    }
    g1_aff a;
    g1_to_aff(&a, &acc);
    fe x, y;
    fe_from_mont(&x, &a.x, &FQ_F);
    fe_from_mont(&y, &a.y, &FQ_F);
    fe_to_words(out, &x);
    fe_to_words(out + 8, &y);
  } else {
    g2_xyzz *ps = (g2_xyzz *)m.partials, acc, sw;
    g2_set_inf(&acc);
    for (int w = windows - 1; w >= 0; w--) {
      for (int k = 0; k < c && w < windows - 1; k++) g2_dbl(&acc, &acc);
      g2_set_inf(&sw);
      for (int k = 0; k < chunks; k++) g2_add(&sw, &sw, &ps[(size_t)w * chunks + k]);
      g2_add(&acc, &acc, &sw);
    }
    g2_aff a;
    g2_to_aff(&a, &acc);
    const fe *cs[4] = {&a.x.a, &a.x.b, &a.y.a, &a.y.b};
    for (int i = 0; i < 4; i++) {
      fe v;
      fe_from_mont(&v, cs[i], &FQ_F);
      fe_to_words(out + 8 * i, &v);
    }
  }
  free(m.partials);
  free((void *)m.bases);
  free(d.digits);
  return 0;
}

/* ---------------------------------------------------------------- generator multiples */
/* [k_i]G for the standard generator of `group` (G1 = (1, 2); G2 = the standard BN254 G2
 * generator), by an 8-bit fixed-base comb, then Montgomery batch inversion per thread. */
static const uint32_t G2_GEN_WORDS[32] = {
  0xd992f6ed, 0x46debd5c, 0xf75edadd, 0x674322d4, 0x5e5c4479, 0x426a0066, 0x121f1e76, 0x1800deef,
  0xaef312c2, 0x97e485b7, 0x35a9e712, 0xf1aa4933, 0x31fb5d25, 0x7260bfb7, 0x920d483a, 0x198e9393,
  0x66fa7daa, 0x4ce6cc01, 0x0c43d37b, 0xe3d1e769, 0x8dcb408f, 0x4aab7180, 0xdb8c6deb, 0x12c85ea5,
  0xd122975b, 0x55acdadc, 0x70b38ef3, 0xbc4b3133, 0x690c3395, 0xec9e99ad, 0x585ff075, 0x090689d0,
};

typedef struct {
  int group, out_mont;
  const uint32_t *k;
  size_t n;
  const void *table; /* [32][256] affine */
  uint32_t *out;
} gen_ctx;

#define GEN_BODY(G, AW, T_, MUL_, INV_, IS_ZERO_, ONE_, COORDS, EMIT)                       \
  do {                                                                                       \
    const G##aff *tab = (const G##aff *)g->table;                                            \
    const size_t block = 1024;                                                                \
    G##xyzz *acc = (G##xyzz *)malloc(sizeof(G##xyzz) * block);                               \
    T_ *pre = (T_ *)malloc(sizeof(T_) * block * 2);                                           \
    for (size_t b0 = lo; b0 < hi; b0 += block) {                                             \
      size_t cnt = hi - b0 < block ? hi - b0 : block;                                        \
      for (size_t j = 0; j < cnt; j++) {                                                     \
        const uint32_t *k = g->k + 8 * (b0 + j);                                             \
        G##set_inf(&acc[j]);                                                                 \
        for (int byte = 0; byte < 32; byte++) {                                              \
          uint32_t d = (k[byte / 4] >> (8 * (byte % 4))) & 255;                               \
          if (d) G##add_aff(&acc[j], &acc[j], &tab[byte * 256 + d]);                          \
        }                                                                                    \
      }                                                                                      \
      /* batch inversion of zz and zzz (infinity: substitute one, emit zeros) */             \
      T_ run = ONE_;                                                                         \
      for (size_t j = 0; j < 2 * cnt; j++) {                                                 \
        const T_ *z = (j & 1) ? &acc[j / 2].zzz : &acc[j / 2].zz;                            \
        pre[j] = run;                                                                        \
        if (!IS_ZERO_(&acc[j / 2].zz)) MUL_(&run, &run, z);                                  \
      }                                                                                      \
      T_ inv;                                                                                \
      INV_(&inv, &run);                                                                      \
      for (size_t j = 2 * cnt; j-- > 0;) {                                                   \
        const T_ *z = (j & 1) ? &acc[j / 2].zzz : &acc[j / 2].zz;                            \
        if (IS_ZERO_(&acc[j / 2].zz)) { pre[j] = inv; continue; }                            \
        T_ zi;                                                                               \
        MUL_(&zi, &inv, &pre[j]);                                                            \
        MUL_(&inv, &inv, z);                                                                 \
        pre[j] = zi;                                                                         \
      }                                                                                      \
      for (size_t j = 0; j < cnt; j++) {                                                     \
        uint32_t *o = g->out + AW * (b0 + j);                                                \
        if (IS_ZERO_(&acc[j].zz)) { memset(o, 0, AW * 4); continue; }                        \
        T_ x, y;                                                                             \
        MUL_(&x, &acc[j].x, &pre[2 * j]);                                                    \
        MUL_(&y, &acc[j].y, &pre[2 * j + 1]);                                                \
        EMIT;                                                                                \
      }                                                                                      \
    }                                                                                        \
    free(acc);                                                                               \
    free(pre);                                                                               \
  } while (0)

static void emit_fe(uint32_t *o, const fe *m, int out_mont) {
  fe v;
  if (out_mont) v = *m; else fe_from_mont(&v, m, &FQ_F);
  fe_to_words(o, &v);
}

static void gen_task(void *p, int tid, int nt) {
  gen_ctx *g = (gen_ctx *)p;
  size_t lo = g->n * tid / nt, hi = g->n * (tid + 1) / nt;
  if (g->group == 1) {
    GEN_BODY(g1_, 16, fe, fq_mul_, fq_inv_, fe_is_zero, FQ_F.one, 2,
             (emit_fe(o, &x, g->out_mont), emit_fe(o + 8, &y, g->out_mont)));
  } else {
    GEN_BODY(g2_, 32, fe2, fe2_mul, fe2_inv, fe2_is_zero, FQ2_ONE, 4,
             (emit_fe(o, &x.a, g->out_mont), emit_fe(o + 8, &x.b, g->out_mont),
              emit_fe(o + 16, &y.a, g->out_mont), emit_fe(o + 24, &y.b, g->out_mont)));
  }
}

/* out[i] = [k_i]G as affine words (plain, or Montgomery-2^256 if out_mont). k_i are reduced
 * 256-bit integers (any value works: the comb uses all 32 bytes). */
int oracle_generator_multiples(int group, const uint32_t *k, size_t n, int threads, int out_mont, uint32_t *out) {
  if (group != 1 && group != 2) return -1;
  if (threads < 1) threads = 1;
  gen_ctx g = {group, out_mont, k, n, NULL, out};
  if (group == 1) {
    g1_aff *tab = (g1_aff *)calloc(32 * 256, sizeof(g1_aff));
    g1_xyzz base, acc;
    fe one = {{1, 0, 0, 0}}, two = {{2, 0, 0, 0}};
    g1_aff gen;
    fe_to_mont(&gen.x, &one, &FQ_F);
    fe_to_mont(&gen.y, &two, &FQ_F);
    g1_from_aff(&base, &gen);
    for (int byte = 0; byte < 32; byte++) {
      g1_set_inf(&acc);
      for (int d = 1; d < 256; d++) {
        g1_add(&acc, &acc, &base);
        g1_to_aff(&tab[byte * 256 + d], &acc);
      }
      for (int s = 0; s < 8; s++) g1_dbl(&base, &base);
    }
    g.table = tab;
    run_parallel(threads, gen_task, &g);
    free(tab);
  } else {
    g2_aff *tab = (g2_aff *)calloc(32 * 256, sizeof(g2_aff));
    g2_xyzz base, acc;
    g2_aff gen;
    fe *cs[4] = {&gen.x.a, &gen.x.b, &gen.y.a, &gen.y.b};
    for (int i = 0; i < 4; i++) {
      fe_from_words(cs[i], G2_GEN_WORDS + 8 * i);
      fe_to_mont(cs[i], cs[i], &FQ_F);
    }
    g2_from_aff(&base, &gen);
    for (int byte = 0; byte < 32; byte++) {
      g2_set_inf(&acc);
      for (int d = 1; d < 256; d++) {
        g2_add(&acc, &acc, &base);
        g2_to_aff(&tab[byte * 256 + d], &acc);
      }
      for (int s = 0; s < 8; s++) g2_dbl(&base, &base);
    }
    g.table = tab;
    run_parallel(threads, gen_task, &g);
    free(tab);
  }
  return 0;
}

/* ---------------------------------------------------------------- Fr helpers */
typedef struct {
  const uint32_t *a, *b;
  size_t n;
  fe *partial;
} dot_ctx;

static void dot_task(void *p, int tid, int nt) {
  dot_ctx *d = (dot_ctx *)p;
  size_t lo = d->n * tid / nt, hi = d->n * (tid + 1) / nt;
  fe acc = {{0, 0, 0, 0}};
  for (size_t i = lo; i < hi; i++) {
    fe x, y, t;
    fe_from_words(&x, d->a + 8 * i);
    fe_from_words(&y, d->b + 8 * i);
    /* values may be >= r: one Montgomery product by R^2 reduces them */
    fe_mul(&x, &x, &FR_F.r2, &FR_F);
    fe_mul(&t, &x, &y, &FR_F); /* x*R * y / R = x*y mod r */
    fe_add(&acc, &acc, &t, &FR_F);
  }
  d->partial[tid] = acc;
}

/* out = sum_i a_i * b_i mod r (plain words). */
void oracle_fr_dot(const uint32_t *a, const uint32_t *b, size_t n, int threads, uint32_t *out) {
  if (threads < 1) threads = 1;
  dot_ctx d = {a, b, n, (fe *)calloc(threads, sizeof(fe))};
  run_parallel(threads, dot_task, &d);
  fe acc = {{0, 0, 0, 0}};
  for (int t = 0; t < threads; t++) fe_add(&acc, &acc, &d.partial[t], &FR_F);
  fe_to_words(out, &acc);
  free(d.partial);
}

/* [k]P for one point (plain affine words in and out). */
void oracle_scalar_mul(int group, const uint32_t *point, const uint32_t *k, uint32_t *out) {
  uint64_t kk[4];
  for (int i = 0; i < 4; i++) kk[i] = (uint64_t)k[2 * i] | ((uint64_t)k[2 * i + 1] << 32);
  if (group == 1) {
    g1_aff *p = (g1_aff *)load_bases(1, point, 0, 1), a;
    g1_xyzz r;
    g1_scalar_mul(&r, p, kk);
    g1_to_aff(&a, &r);
    fe x, y;
    fe_from_mont(&x, &a.x, &FQ_F);
    fe_from_mont(&y, &a.y, &FQ_F);
    fe_to_words(out, &x);
    fe_to_words(out + 8, &y);
    free(p);
  } else {
    g2_aff *p = (g2_aff *)load_bases(2, point, 0, 1), a;
    g2_xyzz r;
    g2_scalar_mul(&r, p, kk);
    g2_to_aff(&a, &r);
    const fe *cs[4] = {&a.x.a, &a.x.b, &a.y.a, &a.y.b};
    for (int i = 0; i < 4; i++) {
      fe v;
      fe_from_mont(&v, cs[i], &FQ_F);
      fe_to_words(out + 8 * i, &v);
    }
    free(p);
  }
}

/* ---------------------------------------------------------------- NTT */
static void fr_root_of_unity(fe *w, int log_n) {
  /* 5^((r-1) >> log_n) (src/host.rs:94-98), Montgomery form */
  uint64_t e[4], one[4] = {1, 0, 0, 0};
  sub4(e, FR_F.p, one);
  for (int s = 0; s < log_n; s++) {
    for (int i = 0; i < 4; i++) e[i] = (e[i] >> 1) | (i < 3 ? e[i + 1] << 63 : 0);
  }
  fe five = {{5, 0, 0, 0}};
  fe_to_mont(&five, &five, &FR_F);
  fe_pow(w, &five, e, &FR_F);
}

typedef struct {
  fe *a;        /* data, Montgomery form */
  fe *tw;       /* w^j, j < n/2, Montgomery form */
  int log_n;
  size_t n;
  int split;    /* stages before the block-local phase */
  pthread_barrier_t *bar;
  fe scale;     /* for inverse: n^-1 (Montgomery) */
  int inverse;
  const uint32_t *in;
  uint32_t *out;
} ntt_ctx;

static inline void butterfly(fe *a, fe *b, const fe *w) {
  fe s, d;
  fe_add(&s, a, b, &FR_F);
  fe_sub(&d, a, b, &FR_F);
  *a = s;
  fe_mul(b, &d, w, &FR_F);
}

static inline size_t bitrev(size_t x, int bits) {
  size_t r = 0;
  for (int i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
  return r;
}

static void ntt_task(void *p, int tid, int nt) {
  ntt_ctx *c = (ntt_ctx *)p;
  size_t n = c->n, half = n / 2;
  /* load + to Montgomery */
  for (size_t i = n * tid / nt; i < n * (tid + 1) / nt; i++) {
    fe_from_words(&c->a[i], c->in + 8 * i);
    fe_to_mont(&c->a[i], &c->a[i], &FR_F);
  }
  /* twiddles: each thread computes its slice from w^lo */
  {
    size_t lo = half * tid / nt, hi = half * (tid + 1) / nt;
    fe w, x;
    fr_root_of_unity(&w, c->log_n);
    if (c->inverse) fe_inv(&w, &w, &FR_F);
    uint64_t e[4] = {lo, 0, 0, 0};
    fe_pow(&x, &w, e, &FR_F);
    for (size_t j = lo; j < hi; j++) { c->tw[j] = x; fe_mul(&x, &x, &w, &FR_F); }
  }
  pthread_barrier_wait(c->bar);
  /* phase 1: the first `split` stages, butterflies split across threads */
  for (int st = 0; st < c->split; st++) {
    size_t h = n >> (st + 1);
    for (size_t b = half * tid / nt; b < half * (tid + 1) / nt; b++) {
      size_t blk = b / h, j = b % h, i = blk * 2 * h + j;
      butterfly(&c->a[i], &c->a[i + h], &c->tw[j << st]);
    }
    pthread_barrier_wait(c->bar);
  }
  /* phase 2: the remaining stages act on independent blocks of 2^(log_n - split) */
  size_t bsize = n >> c->split, blocks = (size_t)1 << c->split;
  for (size_t blk = blocks * tid / nt; blk < blocks * (tid + 1) / nt; blk++) {
    fe *base = c->a + blk * bsize;
    for (int st = c->split; st < c->log_n; st++) {
      size_t h = n >> (st + 1);
      for (size_t g = 0; g < bsize; g += 2 * h)
        for (size_t j = 0; j < h; j++) butterfly(&base[g + j], &base[g + j + h], &c->tw[j << st]);
    }
  }
  pthread_barrier_wait(c->bar);
  /* bit-reversed gather into natural order, scale, back to plain words */
  for (size_t i = n * tid / nt; i < n * (tid + 1) / nt; i++) {
    fe v = c->a[bitrev(i, c->log_n)];
    if (c->inverse) fe_mul(&v, &v, &c->scale, &FR_F);
    fe_from_mont(&v, &v, &FR_F);
    fe_to_words(c->out + 8 * i, &v);
  }
}

/* In-place NTT over Fr of 2^log_n plain elements (8 words each), natural order in and out;
 * the inverse includes the 1/n factor. */
int oracle_ntt(uint32_t *data, int log_n, int inverse, int threads) {
  if (log_n < 1 || log_n > 28) return -1;
  if (threads < 1) threads = 1;
  size_t n = (size_t)1 << log_n;
  if ((size_t)threads > n / 2) threads = (int)(n / 2);
  ntt_ctx c;
  c.a = (fe *)malloc(sizeof(fe) * n);
  c.tw = (fe *)malloc(sizeof(fe) * (n / 2));
  c.log_n = log_n; c.n = n; c.inverse = inverse;
  c.in = data; c.out = data;
  /* block-local once a block of 2^14 elements (512 KB) is reached, but with at least as
   * many blocks as threads */
  int split = log_n > 14 ? log_n - 14 : 0;
  while (((size_t)1 << split) < (size_t)threads && split < log_n) split++;
  c.split = split;
  fe nn = {{n, 0, 0, 0}};
  fe_to_mont(&nn, &nn, &FR_F);
  fe_inv(&c.scale, &nn, &FR_F);
  pthread_barrier_t bar;
  pthread_barrier_init(&bar, NULL, threads);
  c.bar = &bar;
  run_parallel(threads, ntt_task, &c);
  pthread_barrier_destroy(&bar);
  free(c.a);
  free(c.tw);
  return 0;
}

/* One transform output X[k] = sum_i x_i w^(ik) (times 1/n for the inverse), by Horner:
 * O(n) spot check for sizes where the whole transform is too slow to compare. */
void oracle_ntt_eval(const uint32_t *data, int log_n, uint64_t k, int inverse, uint32_t *out) {
  size_t n = (size_t)1 << log_n;
  fe w, x, acc = {{0, 0, 0, 0}};
  fr_root_of_unity(&w, log_n);
  if (inverse) fe_inv(&w, &w, &FR_F);
  uint64_t e[4] = {k, 0, 0, 0};
  fe_pow(&x, &w, e, &FR_F);
  for (size_t i = n; i-- > 0;) {
    fe v;
    fe_from_words(&v, data + 8 * i);
    fe_to_mont(&v, &v, &FR_F);
    fe_mul(&acc, &acc, &x, &FR_F);
    fe_add(&acc, &acc, &v, &FR_F);
  }
  if (inverse) {
    fe nn = {{n, 0, 0, 0}}, ni;
    fe_to_mont(&nn, &nn, &FR_F);
    fe_inv(&ni, &nn, &FR_F);
    fe_mul(&acc, &acc, &ni, &FR_F);
  }
  fe_from_mont(&acc, &acc, &FR_F);
  fe_to_words(out, &acc);
}

/* x_i <- x_i * g^i (plain words in place): the coset shift of the Groth16 witness map. */
void oracle_coset_shift(uint32_t *data, size_t n, const uint32_t *g_words) {
  fe g, x;
  fe_from_words(&g, g_words);
  fe_to_mont(&g, &g, &FR_F);
  x = FR_F.one;
  for (size_t i = 0; i < n; i++) {
    fe v;
    fe_from_words(&v, data + 8 * i);
    fe_mul(&v, &v, &x, &FR_F); /* plain * mont = plain */
    fe_to_words(data + 8 * i, &v);
    fe_mul(&x, &x, &g, &FR_F);
  }
}

/* Montgomery-2^256 <-> plain conversions of Fq coordinates, for building fixtures. */
void oracle_fq_to_mont256(uint32_t *words, size_t count) {
  for (size_t i = 0; i < count; i++) {
    fe v;
    fe_from_words(&v, words + 8 * i);
    fe_to_mont(&v, &v, &FQ_F);
    fe_to_words(words + 8 * i, &v);
  }
}
