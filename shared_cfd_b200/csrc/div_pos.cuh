// div_pos.cuh -- a branch-free quotient for the hot kernels.
#pragma once

namespace scfd {

// a / b for a positive normal b, without branches: the IEEE division's
// out-of-line slow path keeps the many independent quotients of a thread apart,
// these overlap.  Newton-Raphson on the reciprocal from the hardware's
// approximate reciprocal y0 (rcp.approx.ftz, about 23 bits): FP64 takes one
// third-order step y1 = y0 (1 + e + e^2), e = 1 - b y0 (relative error about
// e^3), FP32 one second-order step y1 = y0 (1 + e); then q0 = a y1 and
// Markstein's remainder correction q = q0 + (a - b q0) y1.  The result is
// within one unit in the last place of a / b (tests/test_division.py checks the
// steps in exact arithmetic from seeds 2^-21 off).  A zero, subnormal, infinite
// or negative b is outside its domain; each kernel that uses it states which
// denominators it gives it.
__device__ __forceinline__ double div_pos(double a, double b) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    const double e = fma(-b, y, 1.0);
    y = fma(fma(e, e, e), y, y);
    const double q = a * y;
    return fma(fma(-b, q, a), y, q);
}
__device__ __forceinline__ float div_pos(float a, float b) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
    y = fmaf(fmaf(-b, y, 1.0f), y, y);
    const float q = a * y;
    return fmaf(fmaf(-b, q, a), y, q);
}

}  // namespace scfd
