// Set-up and test helpers (testing.cu).
#pragma once
#include "runtime.hpp"

namespace zkg {

void point_ops(zkg_ctx* ctx, int group, const uint32_t* pairs, size_t count, uint32_t* out);
// Operations per second: variant 0 mad.lo.u32, 1 mad.hi.u32, 2 carry-chained mad.lo.cc /
// madc.hi.cc, 3 Fq Montgomery products, 9 fma.rn.f64, 11 Fq products in FP64 limbs.
double bench_integer_pipe(zkg_ctx* ctx, int variant);
void generator_multiples(zkg_ctx* ctx, int group, const zkg_buf* scalars, size_t n, int mont256, zkg_buf* out);

}  // namespace zkg
