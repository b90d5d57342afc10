// Complex reciprocal of the persistent sweep's Gauss-Jordan pivots (shared
// with the unit test that measures its accuracy against IEEE division).
#pragma once
#include "rgf_internal.cuh"

namespace rgf {

// 1/z = conj(z) r with r = 1/|z|^2 by Newton's iteration for the reciprocal,
// r <- r + r (1 - n r), whose error e = 1 - n r squares at every step
// (Newton's method applied to f(r) = 1/r - n; e.g. Markstein, "IA-64 and
// elementary functions", 2000, ch. 8, for its use in hardware division),
// started from rcp.approx.ftz.f64 and run twice: the result is within a few
// ulp of the correctly rounded 1/n for |z|^2 in the normal double range (a
// unit test measures it).  Branch-free, so every lane of a warp can form it
// speculatively; |z|^2 = 0 or subnormal gives a non-finite result and |z|^2
// above ~2^1022 a zero one, both of which the caller flags as singular.
__device__ __forceinline__ double2 crecip_nr(double2 z) {
  const double n = fma(z.x, z.x, z.y * z.y);
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(n));
  double e = fma(-n, r, 1.0);
  r = fma(r, e, r);
  e = fma(-n, r, 1.0);
  r = fma(r, e, r);
  return cmk(z.x * r, -z.y * r);
}

}  // namespace rgf
