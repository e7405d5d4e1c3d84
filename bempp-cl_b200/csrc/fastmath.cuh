// Sine / cosine pairs for the assembly kernels.
//
// Method: Cody-Waite argument reduction (W. J. Cody and W. Waite, "Software
// Manual for the Elementary Functions", 1980) to a in [-pi/4, pi/4] with
// x = n pi/2 + a, then polynomials in a^2, then the quadrant n mod 4 selects
// and signs the pair.  The reduction constant pi/2 is split into parts with
// few significant bits so that n * part is exact for the n that occur here.
//
// FP64: pi/2 = C1 + C2 + C3 with C1, C2 of 33 significant bits (n * C1 and
// n * C2 exact for |n| < 2^20); then sin a = a + a^3 P(a^2) and
// cos a = 1 + a^2 Q(a^2) with P, Q Chebyshev approximations on |a| <= pi/4
// (degrees 13 and 14 in a; coefficients and error bounds from fit_sincos.py,
// which also fits the reduction-free variants for |x| <= 1 and |x| <= 1/2).
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

// Horner evaluation of sin x = x + x^3 P(x^2) and cos x = 1 + x^2 Q(x^2) with
// the coefficient lists of fit_sincos.py (highest degree first).
template <int NS, int NC>
__device__ __forceinline__ void sincos_poly64(double x, const double (&ps)[NS], const double (&pc)[NC], double *s,
                                              double *c) {
    const double x2 = x * x;
    double p = ps[0];
#pragma unroll
    for (int i = 1; i < NS; ++i) p = fma(p, x2, ps[i]);
    *s = fma(x * x2, p, x);
    double q = pc[0];
#pragma unroll
    for (int i = 1; i < NC; ++i) q = fma(q, x2, pc[i]);
    *c = fma(x2, q, 1.0);
}

// Chebyshev coefficients (fit_sincos.py); maximum absolute errors of the
// polynomials: cw 1.4e-17 / 4.2e-19 on |a| <= pi/4, small 9.0e-18 / 1.1e-17 on
// |x| <= 1, half 3.7e-17 / 5.5e-19 on |x| <= 1/2 (sin / cos).
#define BC_SIN_CW64 {1.5918129294866608e-10, -2.5051131845003624e-08, 2.755731610255244e-06, \
                     -0.00019841269836758574, 0.008333333333330948, -0.16666666666666666}
#define BC_COS_CW64 {-1.1367998654022494e-11, 2.0875886738047052e-09, -2.7557315566341895e-07, \
                     2.480158729369346e-05, -0.0013888888888880775, 0.04166666666666664, -0.5}
#define BC_SIN_SMALL64 {-7.549371704181243e-13, 1.6057701922579786e-10, -2.5052099244914114e-08, \
                        2.755731919201122e-06, -0.00019841269841216566, 0.0083333333333333, -0.16666666666666666}
#define BC_COS_SMALL64 {-1.1304620460700782e-11, 2.0874477943664777e-09, -2.755730370192223e-07, \
                        2.4801587247292686e-05, -0.0013888888888798428, 0.0416666666666661, -0.5}
#define BC_SIN_HALF64 {-2.4951933287704484e-08, 2.755710022606947e-06, -0.0001984126964579005, \
                       0.008333333333272254, -0.16666666666666635}
#define BC_COS_HALF64 {2.0790894217124703e-09, -2.7557077887523167e-07, 2.4801586988836374e-05, \
                       -0.0013888888888705666, 0.041666666666666276, -0.5}

// FP32 minimax coefficients (fit_sincos.py, Lawson's algorithm; highest degree first); maximum
// absolute errors evaluated in float with fused multiply-adds: half 5.6e-8 / 3.7e-8 on |x| <= 1/2,
// small 5.7e-8 / 6.1e-8 on |x| <= 1, cw 3.6e-8 / 5.2e-8 on |a| <= pi/4 (sin / cos).
#define BC_SIN_HALF32 {0.008259795606136322f, -0.16666032373905182f}
#define BC_COS_HALF32 {-0.001377024920657277f, 0.04166495054960251f, -0.4999999403953552f}
#define BC_SIN_SMALL32 {-0.00019283789151813835f, 0.00832979753613472f, -0.16666598618030548f}
#define BC_COS_SMALL32 {2.4138245862559415e-05f, -0.0013883339706808329f, 0.041666481643915176f, \
                        -0.4999999701976776f}
#define BC_SIN_CW32 {-0.000194956359337084f, 0.00833197869360447f, -0.16666650772094727f}
#define BC_COS_CW32 {2.4390450562350452e-05f, -0.0013886763481423259f, 0.04166662320494652f, -0.5f}

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
    constexpr double ps[] = BC_SIN_CW64;
    constexpr double pc[] = BC_COS_CW64;
    double sa, ca;
    sincos_poly64(a, ps, pc, &sa, &ca);
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

// |x| <= 1 without reduction (callers know the bound).
__device__ __forceinline__ void sincos_small64(double x, double *s, double *c) {
    constexpr double ps[] = BC_SIN_SMALL64;
    constexpr double pc[] = BC_COS_SMALL64;
    sincos_poly64(x, ps, pc, s, c);
}

// |x| <= 1/2 without reduction (callers know the bound).
__device__ __forceinline__ void sincos_half64(double x, double *s, double *c) {
    constexpr double ps[] = BC_SIN_HALF64;
    constexpr double pc[] = BC_COS_HALF64;
    sincos_poly64(x, ps, pc, s, c);
}

// |x| <= 1/2 in FP32: degree 5 (sin) and 6 (cos), BC_*_HALF32.
__device__ __forceinline__ void sincos_half32(float x, float *s, float *c) {
    constexpr float ps[] = BC_SIN_HALF32;
    constexpr float pc[] = BC_COS_HALF32;
    const float x2 = x * x;
    *s = fmaf(x * x2, fmaf(ps[0], x2, ps[1]), x);
    *c = fmaf(x2, fmaf(fmaf(pc[0], x2, pc[1]), x2, pc[2]), 1.0f);
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

// |x| <= 1 in FP32: degree 7 (sin) and 8 (cos), BC_*_SMALL32.
__device__ __forceinline__ void sincos_small32(float x, float *s, float *c) {
    constexpr float ps[] = BC_SIN_SMALL32;
    constexpr float pc[] = BC_COS_SMALL32;
    const float x2 = x * x;
    *s = fmaf(x * x2, fmaf(fmaf(ps[0], x2, ps[1]), x2, ps[2]), x);
    *c = fmaf(x2, fmaf(fmaf(fmaf(pc[0], x2, pc[1]), x2, pc[2]), x2, pc[3]), 1.0f);
}

__device__ __forceinline__ void sincos_cw32(float x, float *s, float *c) {
    const float magic = 12582912.0f;  // 1.5 * 2^23
    const float t = fmaf(x, 0.6366197466850281f, magic);
    const float n = t - magic;
    const int q = __float_as_int(t);
    float a = fmaf(-n, 1.5703125f, x);
    a = fmaf(-n, 0.0004838267923332751f, a);
    constexpr float ps[] = BC_SIN_CW32;
    constexpr float pc[] = BC_COS_CW32;
    const float a2 = a * a;
    const float sa = fmaf(a * a2, fmaf(fmaf(ps[0], a2, ps[1]), a2, ps[2]), a);
    const float ca = fmaf(a2, fmaf(fmaf(fmaf(pc[0], a2, pc[1]), a2, pc[2]), a2, pc[3]), 1.0f);
    const float ss = (q & 1) ? ca : sa;
    const float cc = (q & 1) ? sa : ca;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

// exp(i x) for a phase |x| below 1e6 (a centroid distance in units of 1/k, a far-field phase) of the
// mixed-precision kernels:
// Cody-Waite reduction by pi/2 in FP64 (two-part constant), then the FP32 minimax polynomials on
// |a| <= pi/4.  The reduced argument keeps its FP64 accuracy until it is rounded to FP32, so the
// phase is within 1e-7 of exp(i x) for any x in range; the FP32 sums it multiplies carry errors of
// the same size.
__device__ __forceinline__ void phase_reduced32(double x, float *s, float *c) {
    const double magic = 6755399441055744.0;  // 1.5 * 2^52: adding it rounds to an integer
    const double t = fma(x, 0.6366197723675814, magic);
    const double n = t - magic;
    const int q = __double2loint(t);
    double a = fma(-n, 1.5707963267948966, x);
    a = fma(-n, 6.123233995736766e-17, a);
    const float af = (float)a;
    constexpr float ps[] = BC_SIN_CW32;
    constexpr float pc[] = BC_COS_CW32;
    const float a2 = af * af;
    const float sa = fmaf(af * a2, fmaf(fmaf(ps[0], a2, ps[1]), a2, ps[2]), af);
    const float ca = fmaf(a2, fmaf(fmaf(fmaf(pc[0], a2, pc[1]), a2, pc[2]), a2, pc[3]), 1.0f);
    // quadrant q: sin = (s, c, -s, -c), cos = (c, -s, -c, s)
    const float ss = (q & 1) ? ca : sa;
    const float cc = (q & 1) ? sa : ca;
    *s = (q & 2) ? -ss : ss;
    *c = ((q + 1) & 2) ? -cc : cc;
}

// e^{-x} (any real x, |x| below ~700) for the mixed-precision kernels: t = -x log2(e) in FP64, split
// t = n + f with n = rint(t), |f| <= 1/2; 2^f by exp2f in FP32 (relative error ~1e-7, the size of the
// FP32 sums it multiplies) and 2^n built exactly in FP64, so a factor far below the FP32 range stays
// exact in scale.  0 below 2^-1022.
__device__ __forceinline__ double exp_neg_reduced(double x) {
    const double t = -x * 1.4426950408889634;  // log2(e)
    const double n = fmin(rint(t), 1023.0);
    if (n < -1022.0) return 0.0;
    const double two_n = __longlong_as_double((long long)(n + 1023.0) << 52);
    return (double)exp2f((float)(t - n)) * two_n;
}

}  // namespace bc
