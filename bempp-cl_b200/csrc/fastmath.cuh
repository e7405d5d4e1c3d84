// Sine / cosine pairs for the assembly kernels.
//
// Method: Cody-Waite argument reduction (W. J. Cody and W. Waite, "Software
// Manual for the Elementary Functions", 1980) to a in [-pi/4, pi/4] with
// x = n pi/2 + a, then polynomials in a^2, then the quadrant n mod 4 selects
// and signs the pair.  The reduction constant pi/2 is split into parts with
// few significant bits so that n * part is exact for the n that occur here.
//
// FP64: pi/2 = C1 + C2 + C3 with C1, C2 of 33 significant bits (n * C1 and
// n * C2 exact for |n| < 2^20); Taylor series of sin to a^15 and cos to a^16
// (first omitted terms a^17/17! < 5e-17 and a^18/18! < 2e-18 on |a| <= pi/4).
// Arguments with |x| >= 1e6 go to the CUDA library sincos.
//
// FP32: pi/2 = 1.5703125 + 4.838268e-4 (the first part has 8 significant
// bits), and polynomials of degree 7 (sin) and 8 (cos) whose coefficients
// were fitted by weighted least squares on Chebyshev nodes of [-pi/4, pi/4]
// (max abs error 4e-8 / 7e-8 in FP32 arithmetic).  sincos_small32 skips the
// reduction for |x| <= 1 with coefficients fitted on [-1, 1] (max abs error
// 8e-8); callers use it only when a bound on |x| is known.
#pragma once

namespace bc {

__device__ __forceinline__ void sincos_cw64(double x, double *s, double *c) {
    if (!(fabs(x) < 1.0e6)) {
        sincos(x, s, c);
        return;
    }
    const double magic = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
    const double t = fma(x, 0.6366197723675814, magic);
    const double n = t - magic;
    const int q = __double2loint(t);
    double a = fma(-n, 1.5707963267341256, x);
    a = fma(-n, 6.077100506303966e-11, a);
    a = fma(-n, 2.0222662487959506e-21, a);
    const double a2 = a * a;
    double ps = -7.647163731819816e-13;
    ps = fma(ps, a2, 1.6059043836821613e-10);
    ps = fma(ps, a2, -2.505210838544172e-08);
    ps = fma(ps, a2, 2.7557319223985893e-06);
    ps = fma(ps, a2, -0.0001984126984126984);
    ps = fma(ps, a2, 0.008333333333333333);
    ps = fma(ps, a2, -0.16666666666666666);
    const double sa = fma(a * a2, ps, a);
    double pc = 4.779477332387385e-14;
    pc = fma(pc, a2, -1.1470745597729725e-11);
    pc = fma(pc, a2, 2.08767569878681e-09);
    pc = fma(pc, a2, -2.755731922398589e-07);
    pc = fma(pc, a2, 2.48015873015873e-05);
    pc = fma(pc, a2, -0.001388888888888889);
    pc = fma(pc, a2, 0.041666666666666664);
    pc = fma(pc, a2, -0.5);
    const double ca = fma(a2, pc, 1.0);
    // quadrant q: sin = (s, c, -s, -c), cos = (c, -s, -c, s)
    const double ss = (q & 1) ? ca : sa;
    const double cc = (q & 1) ? sa : ca;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

// 1/sqrt(x) in FP64 for finite x > 0: the hardware approximation
// rsqrt.approx.ftz.f64 (relative error below 1e-6; measured 9.1e-7 over
// [1e-300, 1e300]) refined by one step of the third-order iteration
//   y <- y (1 + e/2 + 3 e^2 / 8),  e = 1 - x y^2,
// the binomial series of (1 - e)^(-1/2) = 1 / (y sqrt(x)) truncated after e^2.
// The truncation error (5/16) e^3 is below 1e-17, so the result is within
// rounding (measured maximum relative error 1.37e-16 over the same range).
// Five FP64 operations and no special-case branches: x = 0 or +inf give NaN,
// and subnormal x is flushed to zero.
__device__ __forceinline__ double rsqrt64(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-(x * y), y, 1.0);
    return fma(y * e, fma(0.375, e, 0.5), y);
}

// |x| <= 1 without reduction: Taylor series of sin to x^17 and cos to x^18
// (first omitted terms 1/19! < 9e-18 and 1/20! < 5e-19).
__device__ __forceinline__ void sincos_small64(double x, double *s, double *c) {
    const double x2 = x * x;
    double ps = 2.8114572543455206e-15;
    ps = fma(ps, x2, -7.647163731819816e-13);
    ps = fma(ps, x2, 1.6059043836821613e-10);
    ps = fma(ps, x2, -2.505210838544172e-08);
    ps = fma(ps, x2, 2.7557319223985893e-06);
    ps = fma(ps, x2, -0.0001984126984126984);
    ps = fma(ps, x2, 0.008333333333333333);
    ps = fma(ps, x2, -0.16666666666666666);
    *s = fma(x * x2, ps, x);
    double pc = -1.5619206968586225e-16;
    pc = fma(pc, x2, 4.779477332387385e-14);
    pc = fma(pc, x2, -1.1470745597729725e-11);
    pc = fma(pc, x2, 2.08767569878681e-09);
    pc = fma(pc, x2, -2.755731922398589e-07);
    pc = fma(pc, x2, 2.48015873015873e-05);
    pc = fma(pc, x2, -0.001388888888888889);
    pc = fma(pc, x2, 0.041666666666666664);
    pc = fma(pc, x2, -0.5);
    *c = fma(x2, pc, 1.0);
}

// |x| <= 1/2 without reduction: Taylor series of sin to x^13 and cos to x^14
// (first omitted terms (1/2)^15/15! < 3e-17 and (1/2)^16/16! < 8e-19).
__device__ __forceinline__ void sincos_half64(double x, double *s, double *c) {
    const double x2 = x * x;
    double ps = 1.6059043836821613e-10;
    ps = fma(ps, x2, -2.505210838544172e-08);
    ps = fma(ps, x2, 2.7557319223985893e-06);
    ps = fma(ps, x2, -0.0001984126984126984);
    ps = fma(ps, x2, 0.008333333333333333);
    ps = fma(ps, x2, -0.16666666666666666);
    *s = fma(x * x2, ps, x);
    double pc = -1.1470745597729725e-11;
    pc = fma(pc, x2, 2.08767569878681e-09);
    pc = fma(pc, x2, -2.755731922398589e-07);
    pc = fma(pc, x2, 2.48015873015873e-05);
    pc = fma(pc, x2, -0.001388888888888889);
    pc = fma(pc, x2, 0.041666666666666664);
    pc = fma(pc, x2, -0.5);
    *c = fma(x2, pc, 1.0);
}

// |x| <= 1/2 in FP32: degree 5 (sin) and 6 (cos), coefficients fitted by
// weighted least squares on Chebyshev nodes of [-1/2, 1/2] (max abs error
// 8e-8 / 5e-8 in FP32 arithmetic).
__device__ __forceinline__ void sincos_half32(float x, float *s, float *c) {
    const float x2 = x * x;
    *s = fmaf(x * x2, fmaf(0.008264548145234585f, x2, -0.1666613519191742f), x);
    *c = fmaf(x2, fmaf(fmaf(-0.001377025037072599f, x2, 0.04166495054960251f), x2, -0.4999999403953552f), 1.0f);
}

// Single-instruction FP32 approximations (PTX rsqrt.approx / rcp.approx with
// flush-to-zero; relative error below 2^-22 on normal inputs).  The mixed
// path feeds them squared distances and distance sums of non-adjacent
// elements: positive normal numbers.
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void sincos_small32(float x, float *s, float *c) {
    const float x2 = x * x;
    float ps = fmaf(-0.00019318617705721408f, x2, 0.008330317214131355f);
    ps = fmaf(ps, x2, -0.1666661649942398f);
    *s = fmaf(x * x2, ps, x);
    float pc = fmaf(2.4138245862559415e-05f, x2, -0.0013883339706808329f);
    pc = fmaf(pc, x2, 0.041666481643915176f);
    pc = fmaf(pc, x2, -0.4999999701976776f);
    *c = fmaf(x2, pc, 1.0f);
}

__device__ __forceinline__ void sincos_cw32(float x, float *s, float *c) {
    const float magic = 12582912.0f;  // 1.5 * 2^23
    const float t = fmaf(x, 0.6366197466850281f, magic);
    const float n = t - magic;
    const int q = __float_as_int(t);
    float a = fmaf(-n, 1.5703125f, x);
    a = fmaf(-n, 0.0004838267923332751f, a);
    const float a2 = a * a;
    float ps = fmaf(-0.0001951729936990887f, a2, 0.008332177996635437f);
    ps = fmaf(ps, a2, -0.16666655242443085f);
    const float sa = fmaf(a * a2, ps, a);
    float pc = fmaf(2.4390450562350452e-05f, a2, -0.0013886763481423259f);
    pc = fmaf(pc, a2, 0.04166662320494652f);
    pc = fmaf(pc, a2, -0.5f);
    const float ca = fmaf(a2, pc, 1.0f);
    const float ss = (q & 1) ? ca : sa;
    const float cc = (q & 1) ? sa : ca;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

}  // namespace bc
