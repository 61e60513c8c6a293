// Compensated FP32 summation (Kahan-Babuska steps and TwoSum combination of
// partials), shared by the reduction kernels and the scratch-free row sum.
//
// State (v, c): the true sum is approximately v - c.  Once the running sum
// stops being finite (an infinite term, or overflow) the compensation is
// dropped and the plain value is carried, so such sums give inf, -inf or NaN
// exactly as the reference's sequential loop does (compile.cpp:974-1034,
// cpp.cpp:172-270: `acc = acc + x`), instead of the NaN that (inf - inf)
// inside the compensation would produce.
//
// The files that include this are compiled with -fmad=false: a contracted
// (t - v) - y would lose the rounding error the compensation exists to keep.
#pragma once
#include <math.h>

namespace ltbdev {

// v += x, with the rounding error kept in c
__device__ __forceinline__ void comp_add(float& v, float& c, float x) {
  const float y = x - c;
  const float t = v + y;
  c = isfinite(t) ? (t - v) - y : 0.f;
  v = t;
}

// (v, c) += (bv, bc): TwoSum of the running values, whose rounding error
// joins the compensation terms
__device__ __forceinline__ void comp_combine(float& v, float& c, float bv, float bc) {
  const float s = v + bv;
  if (!isfinite(s)) {
    v = s;
    c = 0.f;
    return;
  }
  const float bp = s - v;
  const float e = (v - (s - bp)) + (bv - bp);
  c = c + bc - e;
  v = s;
}

// the compensated value of (v, c)
__device__ __forceinline__ float comp_value(float v, float c) {
  return isfinite(v) ? v - c : v;
}

}  // namespace ltbdev
