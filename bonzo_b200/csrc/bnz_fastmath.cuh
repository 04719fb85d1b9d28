// bnz_fastmath.cuh -- device arithmetic of the fast build that replaces an
// IEEE division where a quotient within an ulp or two is enough.
#pragma once

// 1/x for normal, finite x: the hardware's approximate reciprocal (PTX
// rcp.approx.ftz.f64, a seed with about 2^-22 relative error) refined by two
// Newton-Raphson steps for f(y) = 1/y - x, y <- y + y (1 - x y), each of
// which squares the relative error; the residual 1 - x y is formed with one
// rounding by a fused multiply-add.  Without the division's special-case
// path it issues a handful of FP64 instructions.
__device__ __forceinline__ double bnz_nr_rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
