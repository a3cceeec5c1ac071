/* BN254 field arithmetic for the C oracle: 4 x u64 limbs, Montgomery radix 2^256.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; never linked into
 * the product library).
 *
 * Restates the reference's host and device field arithmetic:
 *   moduli FQ, FR ....................... src/field.rs:18-20
 *   add_mod / sub_mod / mul_mod / pow ... src/host.rs:27-60
 *   inverse by Fermat ................... src/host.rs:100-102
 *   Fq2 = Fq[u]/(u^2 + 1) ............... src/group.rs:38-48, src/msm.rs:375-387
 * The reference multiplies with 20 x 13-bit limbs and R = 2^260 (src/field.rs:108-130);
 * the radix is internal, so plain values in and out are identical.
 */
#ifndef ZKG_ORACLE_FIELD_H
#define ZKG_ORACLE_FIELD_H
#include <stdint.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef struct { uint64_t v[4]; } fe;          /* one Fq or Fr element */
typedef struct { fe a, b; } fe2;               /* a + b*u, u^2 = -1 */

typedef struct {
  uint64_t p[4];     /* modulus */
  uint64_t inv;      /* -p^-1 mod 2^64 */
  fe r2;             /* 2^512 mod p */
  fe one;            /* 2^256 mod p (Montgomery one) */
} field;

static const field FQ_F = {
  {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
  0x87d20782e4866389ULL,
  {{0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL}},
  {{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}},
};
static const field FR_F = {
  {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
  0xc2e1f593efffffffULL,
  {{0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL}},
  {{0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL}},
};

static inline int fe_is_zero(const fe *a) { return (a->v[0] | a->v[1] | a->v[2] | a->v[3]) == 0; }
static inline int fe_eq(const fe *a, const fe *b) { return memcmp(a, b, sizeof(fe)) == 0; }

static inline int geq4(const uint64_t *a, const uint64_t *b) {
  for (int i = 3; i >= 0; i--) {
    if (a[i] != b[i]) return a[i] > b[i];
  }
  return 1;
}

static inline void sub4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
  u128 br = 0;
  for (int i = 0; i < 4; i++) {
    u128 d = (u128)a[i] - b[i] - br;
    r[i] = (uint64_t)d;
    br = (d >> 64) ? 1 : 0;
  }
}

static inline void fe_add(fe *r, const fe *a, const fe *b, const field *f) {
  u128 c = 0;
  uint64_t t[4];
  for (int i = 0; i < 4; i++) {
    c += (u128)a->v[i] + b->v[i];
    t[i] = (uint64_t)c;
    c >>= 64;
  }
  /* p < 2^254, so the sum never carries out of 256 bits */
  if (geq4(t, f->p)) sub4(t, t, f->p);
  memcpy(r->v, t, 32);
}

static inline void fe_sub(fe *r, const fe *a, const fe *b, const field *f) {
  uint64_t t[4];
  if (geq4(a->v, b->v)) {
    sub4(t, a->v, b->v);
  } else {
    uint64_t d[4];
    sub4(d, f->p, b->v);
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
      c += (u128)a->v[i] + d[i];
      t[i] = (uint64_t)c;
      c >>= 64;
    }
  }
  memcpy(r->v, t, 32);
}

static inline void fe_neg(fe *r, const fe *a, const field *f) {
  if (fe_is_zero(a)) { *r = *a; return; }
  sub4(r->v, f->p, a->v);
}

/* Montgomery product a*b*2^-256 mod p (CIOS). */
static inline void fe_mul(fe *r, const fe *a, const fe *b, const field *f) {
  uint64_t t[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < 4; i++) {
    u128 c = 0;
    for (int j = 0; j < 4; j++) {
      c += (u128)a->v[j] * b->v[i] + t[j];
      t[j] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[4] = (uint64_t)c;
    t[5] = (uint64_t)(c >> 64);
    uint64_t m = t[0] * f->inv;
    c = (u128)m * f->p[0] + t[0];
    c >>= 64;
    for (int j = 1; j < 4; j++) {
      c += (u128)m * f->p[j] + t[j];
      t[j - 1] = (uint64_t)c;
      c >>= 64;
    }
    c += t[4];
    t[3] = (uint64_t)c;
    t[4] = t[5] + (uint64_t)(c >> 64);
  }
  if (t[4] || geq4(t, f->p)) sub4(t, t, f->p);
  memcpy(r->v, t, 32);
}

static inline void fe_to_mont(fe *r, const fe *a, const field *f) { fe_mul(r, a, &f->r2, f); }
static inline void fe_from_mont(fe *r, const fe *a, const field *f) {
  fe one = {{1, 0, 0, 0}};
  fe_mul(r, a, &one, f);
}

/* a^e (Montgomery in, Montgomery out), e a plain 256-bit exponent. */
static inline void fe_pow(fe *r, const fe *a, const uint64_t e[4], const field *f) {
  fe acc = f->one;
  for (int bit = 255; bit >= 0; bit--) {
    fe_mul(&acc, &acc, &acc, f);
    if ((e[bit / 64] >> (bit % 64)) & 1) fe_mul(&acc, &acc, a, f);
  }
  *r = acc;
}

static inline void fe_inv(fe *r, const fe *a, const field *f) {
  uint64_t e[4];
  uint64_t two[4] = {2, 0, 0, 0};
  sub4(e, f->p, two);
  fe_pow(r, a, e, f);
}

/* Plain 8 x u32 words <-> fe (no Montgomery conversion). */
static inline void fe_from_words(fe *r, const uint32_t *w) {
  for (int i = 0; i < 4; i++) r->v[i] = (uint64_t)w[2 * i] | ((uint64_t)w[2 * i + 1] << 32);
}
static inline void fe_to_words(uint32_t *w, const fe *a) {
  for (int i = 0; i < 4; i++) {
    w[2 * i] = (uint32_t)a->v[i];
    w[2 * i + 1] = (uint32_t)(a->v[i] >> 32);
  }
}

/* ---------------------------------------------------------------- Fq2 (u^2 = -1) */
static inline int fe2_is_zero(const fe2 *a) { return fe_is_zero(&a->a) && fe_is_zero(&a->b); }
static inline int fe2_eq(const fe2 *x, const fe2 *y) { return fe_eq(&x->a, &y->a) && fe_eq(&x->b, &y->b); }
static inline void fe2_add(fe2 *r, const fe2 *x, const fe2 *y) {
  fe_add(&r->a, &x->a, &y->a, &FQ_F);
  fe_add(&r->b, &x->b, &y->b, &FQ_F);
}
static inline void fe2_sub(fe2 *r, const fe2 *x, const fe2 *y) {
  fe_sub(&r->a, &x->a, &y->a, &FQ_F);
  fe_sub(&r->b, &x->b, &y->b, &FQ_F);
}
static inline void fe2_neg(fe2 *r, const fe2 *x) {
  fe_neg(&r->a, &x->a, &FQ_F);
  fe_neg(&r->b, &x->b, &FQ_F);
}
/* (a + bu)(c + du) = (ac - bd) + ((a + b)(c + d) - ac - bd)u */
static inline void fe2_mul(fe2 *r, const fe2 *x, const fe2 *y) {
  fe ac, bd, s1, s2, cross;
  fe_mul(&ac, &x->a, &y->a, &FQ_F);
  fe_mul(&bd, &x->b, &y->b, &FQ_F);
  fe_add(&s1, &x->a, &x->b, &FQ_F);
  fe_add(&s2, &y->a, &y->b, &FQ_F);
  fe_mul(&cross, &s1, &s2, &FQ_F);
  fe_sub(&r->a, &ac, &bd, &FQ_F);
  fe_sub(&cross, &cross, &ac, &FQ_F);
  fe_sub(&r->b, &cross, &bd, &FQ_F);
}
/* 1/(a + bu) = (a - bu)/(a^2 + b^2) */
static inline void fe2_inv(fe2 *r, const fe2 *x) {
  fe a2, b2, nrm, ni;
  fe_mul(&a2, &x->a, &x->a, &FQ_F);
  fe_mul(&b2, &x->b, &x->b, &FQ_F);
  fe_add(&nrm, &a2, &b2, &FQ_F);
  fe_inv(&ni, &nrm, &FQ_F);
  fe_mul(&r->a, &x->a, &ni, &FQ_F);
  fe_mul(&nrm, &x->b, &ni, &FQ_F);
  fe_neg(&r->b, &nrm, &FQ_F);
}

/* Field adapters used by the curve template. */
static inline void fq_add_(fe *r, const fe *a, const fe *b) { fe_add(r, a, b, &FQ_F); }
static inline void fq_sub_(fe *r, const fe *a, const fe *b) { fe_sub(r, a, b, &FQ_F); }
static inline void fq_mul_(fe *r, const fe *a, const fe *b) { fe_mul(r, a, b, &FQ_F); }
static inline void fq_neg_(fe *r, const fe *a) { fe_neg(r, a, &FQ_F); }
static inline void fq_inv_(fe *r, const fe *a) { fe_inv(r, a, &FQ_F); }

#endif
