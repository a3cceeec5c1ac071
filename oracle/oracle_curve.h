/* XYZZ group law for the C oracle, instantiated once per coordinate field.
 *
 * TEST INFRASTRUCTURE ONLY.
 *
 * Restates src/shaders/curve.wgsl:22-75 (dbl-2008-s-1, madd-2008-s, add-2008-s with every
 * special case; infinity is ZZ = 0 in XYZZ and (0, 0) in affine form).
 *
 * Before including, define:
 *   P_        name prefix (g1_ / g2_)
 *   T_        coordinate type (fe / fe2)
 *   ADD_ SUB_ MUL_ NEG_ INV_ IS_ZERO_   coordinate operations (r, a, b) / (r, a)
 *   ONE_      Montgomery one of T_
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(P_, name)

typedef struct { T_ x, y; } FN(aff);           /* infinity: x = y = 0 */
typedef struct { T_ x, y, zz, zzz; } FN(xyzz);  /* infinity: zz = 0 */

static inline int FN(aff_is_inf)(const FN(aff) *p) { return IS_ZERO_(&p->x) && IS_ZERO_(&p->y); }
static inline void FN(set_inf)(FN(xyzz) *p) { memset(p, 0, sizeof(*p)); }
static inline int FN(is_inf)(const FN(xyzz) *p) { return IS_ZERO_(&p->zz); }

static inline void FN(from_aff)(FN(xyzz) *r, const FN(aff) *a) {
  if (FN(aff_is_inf)(a)) { FN(set_inf)(r); return; }
  r->x = a->x; r->y = a->y; r->zz = ONE_; r->zzz = ONE_;
}

static void FN(dbl)(FN(xyzz) *r, const FN(xyzz) *p) {
  if (FN(is_inf)(p)) { *r = *p; return; }
  T_ u, v, w, s, x2, m, t, x3, y3;
  ADD_(&u, &p->y, &p->y);
  MUL_(&v, &u, &u);
  MUL_(&w, &u, &v);
  MUL_(&s, &p->x, &v);
  MUL_(&x2, &p->x, &p->x);
  ADD_(&m, &x2, &x2);
  ADD_(&m, &m, &x2);
  MUL_(&x3, &m, &m);
  ADD_(&t, &s, &s);
  SUB_(&x3, &x3, &t);
  SUB_(&t, &s, &x3);
  MUL_(&y3, &m, &t);
  MUL_(&t, &w, &p->y);
  SUB_(&y3, &y3, &t);
  MUL_(&r->zz, &v, &p->zz);
  MUL_(&r->zzz, &w, &p->zzz);
  r->x = x3; r->y = y3;
}

/* r = p + q, q affine (r may alias p). */
static void FN(add_aff)(FN(xyzz) *r, const FN(xyzz) *p, const FN(aff) *q) {
  if (FN(aff_is_inf)(q)) { if (r != p) *r = *p; return; }
  if (FN(is_inf)(p)) { FN(from_aff)(r, q); return; }
  T_ u2, s2, pp, rr, ppsq, ppp, q_, x3, y3, t;
  MUL_(&u2, &q->x, &p->zz);
  MUL_(&s2, &q->y, &p->zzz);
  SUB_(&pp, &u2, &p->x);
  SUB_(&rr, &s2, &p->y);
  if (IS_ZERO_(&pp)) {
    if (IS_ZERO_(&rr)) { FN(dbl)(r, p); } else { FN(set_inf)(r); }
    return;
  }
  MUL_(&ppsq, &pp, &pp);
  MUL_(&ppp, &pp, &ppsq);
  MUL_(&q_, &p->x, &ppsq);
  MUL_(&x3, &rr, &rr);
  SUB_(&x3, &x3, &ppp);
  ADD_(&t, &q_, &q_);
  SUB_(&x3, &x3, &t);
  SUB_(&t, &q_, &x3);
  MUL_(&y3, &rr, &t);
  MUL_(&t, &p->y, &ppp);
  SUB_(&y3, &y3, &t);
  MUL_(&r->zz, &p->zz, &ppsq);
  MUL_(&r->zzz, &p->zzz, &ppp);
  r->x = x3; r->y = y3;
}

/* r = p + q, both XYZZ (r may alias p or q). */
static void FN(add)(FN(xyzz) *r, const FN(xyzz) *p, const FN(xyzz) *q) {
  if (FN(is_inf)(q)) { if (r != p) *r = *p; return; }
  if (FN(is_inf)(p)) { if (r != q) *r = *q; return; }
  T_ u1, u2, s1, s2, pp, rr, ppsq, ppp, q_, x3, y3, t, zz, zzz;
  MUL_(&u1, &p->x, &q->zz);
  MUL_(&u2, &q->x, &p->zz);
  MUL_(&s1, &p->y, &q->zzz);
  MUL_(&s2, &q->y, &p->zzz);
  SUB_(&pp, &u2, &u1);
  SUB_(&rr, &s2, &s1);
  if (IS_ZERO_(&pp)) {
    if (IS_ZERO_(&rr)) { FN(dbl)(r, p); } else { FN(set_inf)(r); }
    return;
  }
  MUL_(&ppsq, &pp, &pp);
  MUL_(&ppp, &pp, &ppsq);
  MUL_(&q_, &u1, &ppsq);
  MUL_(&x3, &rr, &rr);
  SUB_(&x3, &x3, &ppp);
  ADD_(&t, &q_, &q_);
  SUB_(&x3, &x3, &t);
  SUB_(&t, &q_, &x3);
  MUL_(&y3, &rr, &t);
  MUL_(&t, &s1, &ppp);
  SUB_(&y3, &y3, &t);
  MUL_(&zz, &p->zz, &q->zz);
  MUL_(&zz, &zz, &ppsq);
  MUL_(&zzz, &p->zzz, &q->zzz);
  MUL_(&zzz, &zzz, &ppp);
  r->x = x3; r->y = y3; r->zz = zz; r->zzz = zzz;
}

static inline void FN(aff_neg)(FN(aff) *r, const FN(aff) *a) {
  r->x = a->x;
  NEG_(&r->y, &a->y);
}

static void FN(to_aff)(FN(aff) *r, const FN(xyzz) *p) {
  if (FN(is_inf)(p)) { memset(r, 0, sizeof(*r)); return; }
  T_ i;
  INV_(&i, &p->zz);
  MUL_(&r->x, &p->x, &i);
  INV_(&i, &p->zzz);
  MUL_(&r->y, &p->y, &i);
}

/* k * P by double-and-add; k given as 4 plain u64 limbs. */
static void FN(scalar_mul)(FN(xyzz) *r, const FN(aff) *p, const uint64_t k[4]) {
  FN(set_inf)(r);
  for (int bit = 255; bit >= 0; bit--) {
    FN(dbl)(r, r);
    if ((k[bit / 64] >> (bit % 64)) & 1) FN(add_aff)(r, r, p);
  }
}

#undef FN
#undef CAT
#undef CAT2
