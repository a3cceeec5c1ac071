// Host-side XYZZ addition (R = 2^256 Montgomery words), for combining partial MSM results that
// several GPUs computed over shards of the points: add-2008-s and dbl-2008-s-1 (a = 0) as the
// device does them (curve.cuh), over Fq (G1) or Fq2 (G2). Never on the hot path: one addition
// per shard.
#pragma once
#include "host_field.hpp"

namespace zkg::host {

inline U256 e_add(const U256& a, const U256& b) { return add(a, b, fq()); }
inline U256 e_sub(const U256& a, const U256& b) { return sub(a, b, fq()); }
inline U256 e_mul(const U256& a, const U256& b) { return mul(a, b, fq()); }
inline bool e_zero(const U256& a) { return is_zero(a); }
inline U512 e_add(const U512& a, const U512& b) { return U512{add(a.a, b.a, fq()), add(a.b, b.b, fq())}; }
inline U512 e_sub(const U512& a, const U512& b) { return U512{sub(a.a, b.a, fq()), sub(a.b, b.b, fq())}; }
inline U512 e_mul(const U512& a, const U512& b) { return fq2_mul(a, b); }
inline bool e_zero(const U512& a) { return is_zero(a.a) && is_zero(a.b); }

template <class E>
struct XyzzH {
  E x, y, zz, zzz;
};

template <class E>
XyzzH<E> xyzz_double_h(const XyzzH<E>& p) {
  if (e_zero(p.zz)) return p;
  const E u = e_add(p.y, p.y), v = e_mul(u, u), w = e_mul(u, v), s = e_mul(p.x, v);
  const E x2 = e_mul(p.x, p.x), m = e_add(e_add(x2, x2), x2);
  const E x3 = e_sub(e_mul(m, m), e_add(s, s));
  const E y3 = e_sub(e_mul(m, e_sub(s, x3)), e_mul(w, p.y));
  return XyzzH<E>{x3, y3, e_mul(v, p.zz), e_mul(w, p.zzz)};
}

template <class E>
XyzzH<E> xyzz_add_h(const XyzzH<E>& p, const XyzzH<E>& q) {
  if (e_zero(q.zz)) return p;
  if (e_zero(p.zz)) return q;
  const E u1 = e_mul(p.x, q.zz), u2 = e_mul(q.x, p.zz);
  const E s1 = e_mul(p.y, q.zzz), s2 = e_mul(q.y, p.zzz);
  const E pp = e_sub(u2, u1), r = e_sub(s2, s1);
  if (e_zero(pp)) {
    if (e_zero(r)) return xyzz_double_h(p);
    return XyzzH<E>{E{}, E{}, E{}, E{}};
  }
  const E ppsq = e_mul(pp, pp), ppp = e_mul(pp, ppsq), qq = e_mul(u1, ppsq);
  const E x3 = e_sub(e_sub(e_mul(r, r), ppp), e_add(qq, qq));
  const E y3 = e_sub(e_mul(r, e_sub(qq, x3)), e_mul(s1, ppp));
  return XyzzH<E>{x3, y3, e_mul(e_mul(p.zz, q.zz), ppsq), e_mul(e_mul(p.zzz, q.zzz), ppp)};
}

}  // namespace zkg::host
