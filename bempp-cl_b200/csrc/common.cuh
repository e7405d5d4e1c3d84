// Shared device helpers for the bemppcuda kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "../../include/bemppcuda.h"
#include "fastmath.cuh"

#define BC_INV_4PI (0.079577471545947667884441881686257181017229822870228)

namespace bc {

struct cplx {
    double re, im;
};

__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }

// Regular quadrature rule passed by value (lives in the constant parameter bank,
// so kernels use its entries as constant operands without holding registers).
struct QuadRule {
    int nq;
    int pad;
    double x[BEMPPCUDA_MAX_REGULAR_POINTS];
    double y[BEMPPCUDA_MAX_REGULAR_POINTS];
    double w[BEMPPCUDA_MAX_REGULAR_POINTS];
    double sw[BEMPPCUDA_MAX_REGULAR_POINTS][3];  // w times the linear shape values (1 - x - y, x, y)
    float swf[BEMPPCUDA_MAX_REGULAR_POINTS][3];  // sw rounded to FP32 for the mixed path
    float wf[BEMPPCUDA_MAX_REGULAR_POINTS];      // w rounded to FP32 for the mixed path
};

// Number of SMs of the current device (148 on a B200 if the query fails), looked up once per device.
inline int bc_sm_count() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int sms = cached[dev].load(std::memory_order_relaxed);
    if (sms <= 0) {
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
        cached[dev].store(sms, std::memory_order_relaxed);
    }
    return sms;
}

// The first nq points (x, y pairs) and weights of a host rule; unused entries are zero.
inline void fill_rule(QuadRule &rule, int nq, const double *points, const double *weights) {
    rule.nq = nq;
    rule.pad = 0;
    for (int i = 0; i < BEMPPCUDA_MAX_REGULAR_POINTS; ++i) {
        rule.x[i] = i < nq ? points[2 * i] : 0.0;
        rule.y[i] = i < nq ? points[2 * i + 1] : 0.0;
        rule.w[i] = i < nq ? weights[i] : 0.0;
        rule.sw[i][0] = rule.w[i] * (1.0 - rule.x[i] - rule.y[i]);
        rule.sw[i][1] = rule.w[i] * rule.x[i];
        rule.sw[i][2] = rule.w[i] * rule.y[i];
        for (int k = 0; k < 3; ++k) rule.swf[i][k] = (float)rule.sw[i][k];
        rule.wf[i] = (float)rule.w[i];
    }
}

// Geometry of one element read from the field-major record.
struct Geom {
    double v0[3], j0[3], j1[3], n[3];
    double ie;
};

__device__ __forceinline__ void load_geom(const double *__restrict__ g, int64_t ne, int64_t e, double nm, Geom &out) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        out.v0[d] = __ldg(g + (0 + d) * ne + e);
        out.j0[d] = __ldg(g + (3 + d) * ne + e);
        out.j1[d] = __ldg(g + (6 + d) * ne + e);
        out.n[d] = __ldg(g + (9 + d) * ne + e) * nm;
    }
    out.ie = __ldg(g + 12 * ne + e);
}

__device__ __forceinline__ void to_global(const Geom &g, double x, double y, double out[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = fma(g.j1[d], y, fma(g.j0[d], x, g.v0[d]));
}

__device__ __forceinline__ double edge_length(const double *__restrict__ g, int64_t ne, int64_t e, int i) {
    return __ldg(g + (13 + i) * ne + e);
}

// Surface curls (numba_kernels.py:1120-1142): row i = n x (J (J^T J)^-1 grad_ref_i),
// grad_ref = [[-1, 1, 0], [-1, 0, 1]]; n carries the normal multiplier.
__device__ __forceinline__ void surface_curls(const double *__restrict__ g, int64_t ne, int64_t e, const double n[3],
                                              double curl[3][3]) {
    const double gr0[3] = {-1.0, 1.0, 0.0};
    const double gr1[3] = {-1.0, 0.0, 1.0};
    double jit[3][2];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        jit[d][0] = __ldg(g + (16 + 2 * d) * ne + e);
        jit[d][1] = __ldg(g + (17 + 2 * d) * ne + e);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        double sg[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) sg[d] = jit[d][0] * gr0[i] + jit[d][1] * gr1[i];
        curl[i][0] = n[1] * sg[2] - n[2] * sg[1];
        curl[i][1] = n[2] * sg[0] - n[0] * sg[2];
        curl[i][2] = n[0] * sg[1] - n[1] * sg[0];
    }
}

// Piola-mapped RWG functions J r_i / |J| with r = (x, y-1), (x-1, y), (x, y)
// (numba_kernels.py:96-111, shapesets.py:95-102).
__device__ __forceinline__ void rwg_values(const Geom &g, double x, double y, double b[3][3]) {
    const double rx[3] = {x, x - 1.0, x};
    const double ry[3] = {y - 1.0, y, y};
    const double inv = 1.0 / g.ie;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) b[i][d] = (g.j0[d] * rx[i] + g.j1[d] * ry[i]) * inv;
}

__device__ __forceinline__ void scalar_shape(int nshape, double x, double y, double out[3]) {
    if (nshape == 1) {
        out[0] = 1.0;
        out[1] = 0.0;
        out[2] = 0.0;
    } else {
        out[0] = 1.0 - x - y;
        out[1] = x;
        out[2] = y;
    }
}

// Green's functions in FP64 (numba_kernels.py:176-551).  x: test point,
// y: trial point, nx / ny: test / trial normals, p: parameters.  Sine and
// cosine pairs come from sincos_cw64 (fastmath.cuh).
template <int K>
__device__ __forceinline__ cplx greens(const double x[3], const double y[3], const double nx[3], const double ny[3],
                                       const double p[4]) {
    double d0 = y[0] - x[0], d1 = y[1] - x[1], d2 = y[2] - x[2];
    double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
    double rinv = rsqrt64(r2);
    double r = r2 * rinv;
    if (K == BEMPPCUDA_LAPLACE_SLP) {
        return {BC_INV_4PI * rinv, 0.0};
    } else if (K == BEMPPCUDA_LAPLACE_DLP) {
        double dot = fma(d2, ny[2], fma(d1, ny[1], d0 * ny[0]));
        return {-dot * BC_INV_4PI * rinv * rinv * rinv, 0.0};
    } else if (K == BEMPPCUDA_LAPLACE_ADLP) {
        double dot = fma(d2, nx[2], fma(d1, nx[1], d0 * nx[0]));
        return {dot * BC_INV_4PI * rinv * rinv * rinv, 0.0};
    } else if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
        double s, c;
        sincos_cw64(p[0] * r, &s, &c);
        double f = BC_INV_4PI * rinv;
        if (p[1] != 0.0) f *= exp(-p[1] * r);
        return {c * f, s * f};
    } else if (K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP) {
        double dot = (K == BEMPPCUDA_HELMHOLTZ_DLP) ? fma(d2, ny[2], fma(d1, ny[1], d0 * ny[0]))
                                                    : -fma(d2, nx[2], fma(d1, nx[1], d0 * nx[0]));
        double lg = dot * BC_INV_4PI * rinv * rinv * rinv;
        double s, c;
        sincos_cw64(p[0] * r, &s, &c);
        if (p[1] != 0.0) lg *= exp(-p[1] * r);
        double fr = c * lg, fi = s * lg;
        double a = -1.0 - p[1] * r, b = p[0] * r;
        return {a * fr - b * fi, b * fr + a * fi};
    } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
        // DLP + eta SLP: e^{ikr}/(4 pi r) [ (ikr - 1)(y-x).n_y / r^2 + eta ]
        double dot = fma(d2, ny[2], fma(d1, ny[1], d0 * ny[0]));
        double s, c;
        sincos_cw64(p[0] * r, &s, &c);
        double f = BC_INV_4PI * rinv;
        if (p[1] != 0.0) f *= exp(-p[1] * r);
        const double g = dot * rinv * rinv;
        const double ar = (-1.0 - p[1] * r) * g + p[2], ai = p[0] * r * g + p[3];
        const double er = c * f, ei = s * f;
        return {er * ar - ei * ai, er * ai + ei * ar};
    } else if (K == BEMPPCUDA_MODHELM_SLP) {
        return {BC_INV_4PI * exp(-p[0] * r) * rinv, 0.0};
    } else if (K == BEMPPCUDA_MODHELM_DLP) {
        double dot = fma(d2, ny[2], fma(d1, ny[1], d0 * ny[0]));
        return {dot * (-p[0] * r - 1.0) * BC_INV_4PI * exp(-p[0] * r) * rinv * rinv * rinv, 0.0};
    } else if (K == BEMPPCUDA_MODHELM_ADLP) {
        double dot = fma(d2, nx[2], fma(d1, nx[1], d0 * nx[0]));
        return {dot * (p[0] * r + 1.0) * BC_INV_4PI * exp(-p[0] * r) * rinv * rinv * rinv, 0.0};
    } else if (K == BEMPPCUDA_FARFIELD_SLP) {
        double dot = fma(x[2], y[2], fma(x[1], y[1], x[0] * y[0]));
        double s, c;
        sincos_cw64(-p[0] * dot, &s, &c);
        return {BC_INV_4PI * c, BC_INV_4PI * s};
    } else {  // BEMPPCUDA_FARFIELD_DLP
        double dot = fma(x[2], y[2], fma(x[1], y[1], x[0] * y[0]));
        double factor = -p[0] * fma(x[2], ny[2], fma(x[1], ny[1], x[0] * ny[0]));
        double s, c;
        sincos_cw64(-p[0] * dot, &s, &c);
        return {-factor * BC_INV_4PI * s, factor * BC_INV_4PI * c};
    }
}

__device__ __forceinline__ bool share_vertex(const int32_t *__restrict__ el, int64_t a, int64_t b) {
    int a0 = __ldg(el + 3 * a), a1 = __ldg(el + 3 * a + 1), a2 = __ldg(el + 3 * a + 2);
    int b0 = __ldg(el + 3 * b), b1 = __ldg(el + 3 * b + 1), b2 = __ldg(el + 3 * b + 2);
    return a0 == b0 || a0 == b1 || a0 == b2 || a1 == b0 || a1 == b1 || a1 == b2 || a2 == b0 || a2 == b1 ||
           a2 == b2;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace bc

// Host-side error reporting shared by the entry points.
void bc_set_error(const char *fmt, ...);
int bc_check_launch(const char *what);
