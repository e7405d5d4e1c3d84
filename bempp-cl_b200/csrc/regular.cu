// Regular (non-adjacent) element-pair quadrature for dense Galerkin assembly.
//
// Replaces the regular assemblers of bempp_cl/core/numba_kernels.py:
// default_scalar_regular_kernel (:980-1074), laplace/helmholtz/modified
// hypersingular_regular (:1078-1467), maxwell_efield_regular_assembler
// (:1853-1970) and maxwell_mfield_regular_assembler (:2151-2278).
//
// Two kernels:
//  * regular_dp0<K, MIXED>: piecewise-constant test and trial spaces with the
//    identity dof map, 6-point rule.  One thread owns one trial element
//    (a matrix column) and sweeps a block of test elements (rows) staged in
//    shared memory; the 6 trial quadrature points stay in registers; every
//    matrix entry is written exactly once (coalesced along the row).
//    MIXED evaluates the 36 quadrature-point pairs in FP32 relative to the
//    element centroids: the centroid distance r_c and exp(i k r_c) are FP64,
//    per point only the offset r - r_c = (2 D.e + e.e) / (r + r_c) enters
//    the FP32 phase, so the phase error stays ~1e-7 rad independently of
//    k r.  The 6-point inner sums are FP32, the per-entry sum is FP64.
//  * regular_generic<ASM, K>: any scalar / hypersingular / Maxwell
//    assembly with 1 or 3 shape functions and any rule (<= 16 points).  One
//    thread per element pair; the local nshape x nshape block is scattered
//    with atomicAdd into the (pre-zeroed or accumulating) result.
#include <cstdio>

#include "common.cuh"
#include "fastmath.cuh"

namespace bc {

struct RegParams {
    const double *tg;  // test geometry record
    const double *sg;  // trial geometry record
    int64_t tne, sne;
    const int32_t *tel;  // test element vertex ids (ne, 3)
    const int32_t *sel;
    const uint32_t *tsup;
    const uint32_t *ssup;
    int64_t ntest, ntrial;
    const uint32_t *tl2g, *sl2g;
    const double *tmult, *smult;
    const int32_t *tnm, *snm;
    int tnshape, snshape;
    int grids_identical;
    int is_complex;
    int overwrite;
    int pad;
    double p[4];
    void *result;
    int64_t ld;
};

constexpr int DP0_THREADS = 128;
constexpr int DP0_TCHUNK = 32;
constexpr int NQ6 = 6;

// --------------------------------------------------------------------------------------------
// DP0 fast path
// --------------------------------------------------------------------------------------------
// Kernel classes of the fast path.  dotv is (y-x).n_y for double layers and
// -(y-x).n_x for adjoint double layers, so one formula serves both.
template <int K>
struct KernelTraits {
    static constexpr bool helm = (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                                  K == BEMPPCUDA_HELMHOLTZ_ADLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool modhelm = (K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP ||
                                     K == BEMPPCUDA_MODHELM_ADLP);
    static constexpr bool adjoint = (K == BEMPPCUDA_LAPLACE_ADLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
                                     K == BEMPPCUDA_MODHELM_ADLP);
    static constexpr bool dlp = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                                 K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool normal = adjoint || dlp;
    static constexpr bool complex_out = helm;
};

// Stage a block of test elements in shared memory.
struct TestBlock64 {
    double x[DP0_TCHUNK][NQ6][3];
    double c[DP0_TCHUNK][3];
    double n[DP0_TCHUNK][3];
    double ie[DP0_TCHUNK];
    int v[DP0_TCHUNK][3];
};

struct TestBlock32 {
    float4 o[DP0_TCHUNK][NQ6];  // point offset from the centroid, |offset|^2
    double c[DP0_TCHUNK][3];    // centroid
    float n[DP0_TCHUNK][3];
    double ie[DP0_TCHUNK];
    int v[DP0_TCHUNK][3];
};

__device__ __forceinline__ bool shares_vertex(const int *a, int b0, int b1, int b2) {
    return (a[0] == b0) | (a[0] == b1) | (a[0] == b2) | (a[1] == b0) | (a[1] == b1) | (a[1] == b2) | (a[2] == b0) |
           (a[2] == b1) | (a[2] == b2);
}

__device__ __forceinline__ void store_entry(const RegParams &prm, int64_t row, int64_t col, bool adj, double re,
                                            double im) {
    if (prm.is_complex) {
        double2 *out = reinterpret_cast<double2 *>(prm.result) + row * prm.ld + col;
        if (prm.overwrite) {
            *out = make_double2(re, im);
        } else if (!adj) {
            const double2 old = *out;
            *out = make_double2(old.x + re, old.y + im);
        }
    } else {
        double *out = reinterpret_cast<double *>(prm.result) + row * prm.ld + col;
        if (prm.overwrite)
            *out = re;
        else if (!adj)
            *out += re;
    }
}

// FP64: one thread per (trial element, block of 32 test elements).
// CK: the wavenumber has a nonzero imaginary part.
// PHC > 0: |k| (R_t + R_s) <= 1 (class 1) or <= 1/2 (class 2), so
// exp(i k r) = exp(i k r_c) exp(i k (r - r_c)) with r_c the centroid
// distance: the first factor once per element pair, the second from a
// polynomial without range reduction (r - r_c is exact to ~1e-16 r in FP64,
// so no cancellation concern here).  PHC = 0 reduces every argument.
template <int K, bool CK, int PHC>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_fp64(RegParams prm, QuadRule rule) {
    using T = KernelTraits<K>;
    constexpr bool PH = PHC > 0 && T::helm && !CK;  // phase factored about the centroids
    __shared__ TestBlock64 sb;
    const int64_t t0 = (int64_t)blockIdx.y * DP0_TCHUNK;
    const int tcount = (int)min((int64_t)DP0_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        for (int p = 0; p < NQ6; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
#pragma unroll
            for (int d = 0; d < 3; ++d) sb.x[idx][p][d] = x[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.n[idx][d] = g.n[d];
            sb.c[idx][d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        sb.ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3] = {0.0, 0.0, 0.0};
    if (PH)
#pragma unroll
        for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    double y[NQ6][3];
#pragma unroll
    for (int q = 0; q < NQ6; ++q) to_global(gs, rule.x[q], rule.y[q], y[q]);
    const double kr = prm.p[0], ki = prm.p[1], etar = prm.p[2], etai = prm.p[3];
    // normal term (y_q - x_p).n split as (y_q - c).n + (c - x_p).n about the
    // trial element's vertex 0 (both parts well conditioned)
    double ynv[NQ6];
    if (T::normal && !T::adjoint)
#pragma unroll
        for (int q = 0; q < NQ6; ++q)
            ynv[q] = fma(y[q][2] - gs.v0[2], gs.n[2], fma(y[q][1] - gs.v0[1], gs.n[1], (y[q][0] - gs.v0[0]) * gs.n[0]));

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        const bool adj = prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2);
        double acc_re = 0.0, acc_im = 0.0;
        if (!adj) {
            double nv[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) nv[d] = T::adjoint ? sb.n[tt][d] : gs.n[d];
            double rc = 0.0, ph_s = 0.0, ph_c = 1.0;
            if (PH) {
                const double D0 = sc[0] - sb.c[tt][0], D1 = sc[1] - sb.c[tt][1], D2 = sc[2] - sb.c[tt][2];
                rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
                sincos_cw64(kr * rc, &ph_s, &ph_c);
            }
            for (int p = 0; p < NQ6; ++p) {
                const double x0 = sb.x[tt][p][0], x1 = sb.x[tt][p][1], x2 = sb.x[tt][p][2];
                double xn = 0.0;
                if (T::normal && !T::adjoint)
                    xn = fma(gs.v0[2] - x2, nv[2], fma(gs.v0[1] - x1, nv[1], (gs.v0[0] - x0) * nv[0]));
                double sr = 0.0, sim = 0.0, s1r = 0.0, s1i = 0.0;
#pragma unroll
                for (int q = 0; q < NQ6; ++q) {
                    const double d0 = y[q][0] - x0, d1 = y[q][1] - x1, d2 = y[q][2] - x2;
                    const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                    const double rinv = rsqrt(r2);
                    const double wq = rule.w[q];
                    double dotv = 0.0;
                    if (T::normal) {
                        if (T::adjoint)
                            dotv = -fma(d2, nv[2], fma(d1, nv[1], d0 * nv[0]));
                        else
                            dotv = ynv[q] + xn;
                    }
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        sr = fma(wq, rinv, sr);
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        sr = fma(-wq * dotv, rinv * rinv * rinv, sr);
                    } else if (T::modhelm) {
                        const double r = r2 * rinv;
                        const double e = exp(-kr * r);
                        if (K == BEMPPCUDA_MODHELM_SLP)
                            sr = fma(wq * e, rinv, sr);
                        else
                            sr = fma(wq * dotv * (-kr * r - 1.0) * e, rinv * rinv * rinv, sr);
                    } else {  // Helmholtz family
                        const double r = r2 * rinv;
                        double sn, cs;
                        if (PH && PHC == 2)
                            sincos_half64(kr * (r - rc), &sn, &cs);
                        else if (PH)
                            sincos_small64(kr * (r - rc), &sn, &cs);
                        else
                            sincos_cw64(kr * r, &sn, &cs);
                        double f = wq * rinv;
                        if (CK) {
                            f *= exp(-ki * r);
                            const double cf = cs * f, sf = sn * f;
                            if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
                                sr += cf;
                                sim += sf;
                            } else {
                                // (i k r - 1) dotv / r^2 (+ eta)
                                const double v = dotv * rinv;
                                const double u = v * rinv;
                                double a = fma(-ki, v, -u);
                                double b = kr * v;
                                if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                                    a += etar;
                                    b += etai;
                                }
                                sr = fma(cf, a, fma(-sf, b, sr));
                                sim = fma(cf, b, fma(sf, a, sim));
                            }
                        } else {
                            // s0 = sum f e^{ikr} (single-layer part), s1 = sum f v (i k - 1/r) e^{ikr}
                            if (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                                sr = fma(f, cs, sr);
                                sim = fma(f, sn, sim);
                            }
                            if (K != BEMPPCUDA_HELMHOLTZ_SLP) {
                                const double g = f * dotv * rinv;
                                s1r = fma(g, fma(rinv, cs, kr * sn), s1r);
                                s1i = fma(g, fma(kr, cs, -rinv * sn), s1i);
                            }
                        }
                    }
                }
                if (T::helm && !CK && K != BEMPPCUDA_HELMHOLTZ_SLP) {
                    // DLP: -s1r + i s1i; combined: eta * s0 - s1r + i s1i
                    if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                        const double a0 = sr, b0 = sim;
                        sr = fma(etar, a0, fma(-etai, b0, -s1r));
                        sim = fma(etar, b0, fma(etai, a0, s1i));
                    } else {
                        sr = -s1r;
                        sim = s1i;
                    }
                }
                acc_re = fma(rule.w[p], sr, acc_re);
                acc_im = fma(rule.w[p], sim, acc_im);
            }
            const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
            if (PH) {
                const double re = acc_re * ph_c - acc_im * ph_s;
                acc_im = (acc_re * ph_s + acc_im * ph_c) * scale;
                acc_re = re * scale;
            } else {
                acc_re *= scale;
                acc_im *= scale;
            }
        }
        store_entry(prm, row, si, adj, acc_re, acc_im);
    }
}

// Mixed precision: per element pair the centroid offset D = c_s - c_t, its
// length r_c and exp(i k r_c) are FP64; per quadrature-point pair the FP32
// offsets o_p = x_p - c_t, yo_q = y_q - c_s give
//   r^2 - r_c^2 = |yo_q|^2 + 2 D.yo_q + |o_p|^2 - 2 D.o_p - 2 yo_q.o_p
// (the first two terms per trial point, the next two per test point, one
// dot product per pair of points), r from rsqrtf, and the phase offset
// delta = r - r_c = (r^2 - r_c^2) / (r + r_c) without cancellation.
// PHC: 1 or 2 when |k| * (R_t + R_s) <= 1 or <= 1/2 is guaranteed by the
// caller, so the phase k * delta needs no range reduction; 0 reduces it.
template <int K, bool CK, int PHC>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_mixed(RegParams prm, QuadRule rule) {
    using T = KernelTraits<K>;
    __shared__ TestBlock32 sb;
    const int64_t t0 = (int64_t)blockIdx.y * DP0_TCHUNK;
    const int tcount = (int)min((int64_t)DP0_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        double c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) c[d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
        for (int p = 0; p < NQ6; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
            const float o0 = (float)(x[0] - c[0]), o1 = (float)(x[1] - c[1]), o2 = (float)(x[2] - c[2]);
            sb.o[idx][p] = make_float4(o0, o1, o2, fmaf(o2, o2, fmaf(o1, o1, o0 * o0)));
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.c[idx][d] = c[d];
            sb.n[idx][d] = (float)g.n[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        sb.ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    float yo[NQ6][3], yy[NQ6], yn[NQ6];
    const float sn0 = (float)gs.n[0], sn1 = (float)gs.n[1], sn2 = (float)gs.n[2];
#pragma unroll
    for (int q = 0; q < NQ6; ++q) {
        double v[3];
        to_global(gs, rule.x[q], rule.y[q], v);
        yo[q][0] = (float)(v[0] - sc[0]);
        yo[q][1] = (float)(v[1] - sc[1]);
        yo[q][2] = (float)(v[2] - sc[2]);
        yy[q] = fmaf(yo[q][2], yo[q][2], fmaf(yo[q][1], yo[q][1], yo[q][0] * yo[q][0]));
        yn[q] = fmaf(yo[q][2], sn2, fmaf(yo[q][1], sn1, yo[q][0] * sn0));
    }
    const double kr = prm.p[0], ki = prm.p[1];
    const float krf = (float)kr, kif = (float)ki;
    const float etar = (float)prm.p[2], etai = (float)prm.p[3];

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        const bool adj = prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2);
        double acc_re = 0.0, acc_im = 0.0;
        if (!adj) {
            const double D0 = sc[0] - sb.c[tt][0], D1 = sc[1] - sb.c[tt][1], D2 = sc[2] - sb.c[tt][2];
            const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
            const double rc = sqrt(rc2);
            double ph_s = 0.0, ph_c = 1.0, damp = 1.0;
            if (T::helm) {
                sincos_cw64(kr * rc, &ph_s, &ph_c);
                if (CK) damp = exp(-ki * rc);
            } else if (T::modhelm) {
                damp = exp(-kr * rc);
            }
            const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
            const float rcf = (float)rc, rc2f = (float)rc2;
            // normal of the dot product and its trial-side part
            float nx0 = sn0, nx1 = sn1, nx2 = sn2;
            float ynq[NQ6];
            if (T::adjoint) {
                nx0 = sb.n[tt][0];
                nx1 = sb.n[tt][1];
                nx2 = sb.n[tt][2];
#pragma unroll
                for (int q = 0; q < NQ6; ++q) ynq[q] = fmaf(yo[q][2], nx2, fmaf(yo[q][1], nx1, yo[q][0] * nx0));
            } else {
#pragma unroll
                for (int q = 0; q < NQ6; ++q) ynq[q] = yn[q];
            }
            const float Dn = fmaf(D2f, nx2, fmaf(D1f, nx1, D0f * nx0));
            float A[NQ6];
#pragma unroll
            for (int q = 0; q < NQ6; ++q)
                A[q] = fmaf(2.f, fmaf(D2f, yo[q][2], fmaf(D1f, yo[q][1], D0f * yo[q][0])), yy[q]);
            double a64r = 0.0, a64i = 0.0;
            for (int p = 0; p < NQ6; ++p) {
                const float4 o = sb.o[tt][p];
                const float Bp = fmaf(-2.f, fmaf(D2f, o.z, fmaf(D1f, o.y, D0f * o.x)), o.w);
                const float cp = Dn - fmaf(o.z, nx2, fmaf(o.y, nx1, o.x * nx0));
                float sr = 0.f, sim = 0.f;
#pragma unroll
                for (int q = 0; q < NQ6; ++q) {
                    const float ey = fmaf(yo[q][2], o.z, fmaf(yo[q][1], o.y, yo[q][0] * o.x));
                    const float sdot = fmaf(-2.f, ey, A[q] + Bp);  // r^2 - r_c^2
                    const float r2 = rc2f + sdot;
                    const float rinv = rsqrt_approx(r2);
                    const float r = r2 * rinv;
                    const float delta = sdot * rcp_approx(r + rcf);
                    float dotv = 0.f;
                    if (T::normal) {
                        dotv = cp + ynq[q];
                        if (T::adjoint) dotv = -dotv;
                    }
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        sr = fmaf(rule.wf[q], rinv, sr);
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        sr = fmaf(-rule.wf[q] * dotv, rinv * rinv * rinv, sr);
                    } else if (T::modhelm) {
                        const float e = __expf(-krf * delta);
                        if (K == BEMPPCUDA_MODHELM_SLP)
                            sr = fmaf(rule.wf[q] * e, rinv, sr);
                        else
                            sr = fmaf(rule.wf[q] * dotv * (-krf * r - 1.f) * e, rinv * rinv * rinv, sr);
                    } else {
                        float sn, cs;
                        if (PHC == 2)
                            sincos_half32(krf * delta, &sn, &cs);
                        else if (PHC == 1)
                            sincos_small32(krf * delta, &sn, &cs);
                        else
                            sincos_cw32(krf * delta, &sn, &cs);
                        float f = rule.wf[q] * rinv;
                        if (CK) f *= __expf(-kif * delta);
                        const float cf = cs * f, sf = sn * f;
                        if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
                            sr += cf;
                            sim += sf;
                        } else {
                            const float v = dotv * rinv;
                            const float u = v * rinv;
                            float a = CK ? fmaf(-kif, v, -u) : -u;
                            float b = krf * v;
                            if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                                a += etar;
                                b += etai;
                            }
                            sr = fmaf(cf, a, fmaf(-sf, b, sr));
                            sim = fmaf(cf, b, fmaf(sf, a, sim));
                        }
                    }
                }
                a64r = fma(rule.w[p], (double)sr, a64r);
                a64i = fma(rule.w[p], (double)sim, a64i);
            }
            a64r *= damp;
            a64i *= damp;
            const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
            acc_re = (a64r * ph_c - a64i * ph_s) * scale;
            acc_im = (a64r * ph_s + a64i * ph_c) * scale;
        }
        store_entry(prm, row, si, adj, acc_re, acc_im);
    }
}

// Packed mixed precision (Blackwell paired FP32): the same arithmetic as
// regular_dp0_mixed, but trial points q and q+1 travel together through
// fma/add/mul.rn.f32x2, halving the issue slots of the FP32 work; only the
// reciprocal square root and reciprocal stay scalar (one MUFU each).
// Laplace and Helmholtz families with a real wavenumber.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 b2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <int PHC>
__device__ __forceinline__ void sincos2(float2 x, float2 *s, float2 *c) {
    if (PHC == 2) {
        const float2 x2 = mul2(x, x);
        *s = fma2(mul2(x, x2), fma2(b2(0.008264548145234585f), x2, b2(-0.1666613519191742f)), x);
        *c = fma2(x2, fma2(fma2(b2(-0.001377025037072599f), x2, b2(0.04166495054960251f)), x2, b2(-0.4999999403953552f)),
                  b2(1.0f));
    } else if (PHC == 1) {
        const float2 x2 = mul2(x, x);
        float2 ps = fma2(b2(-0.00019318617705721408f), x2, b2(0.008330317214131355f));
        ps = fma2(ps, x2, b2(-0.1666661649942398f));
        *s = fma2(mul2(x, x2), ps, x);
        float2 pc = fma2(b2(2.4138245862559415e-05f), x2, b2(-0.0013883339706808329f));
        pc = fma2(pc, x2, b2(0.041666481643915176f));
        pc = fma2(pc, x2, b2(-0.4999999701976776f));
        *c = fma2(x2, pc, b2(1.0f));
    } else {
        sincos_cw32(x.x, &s->x, &c->x);
        sincos_cw32(x.y, &s->y, &c->y);
    }
}

template <int K, int PHC>
__global__ void __launch_bounds__(DP0_THREADS, 5) regular_dp0_mixed2(RegParams prm, QuadRule rule) {
    using T = KernelTraits<K>;
    constexpr int NP = NQ6 / 2;
    __shared__ TestBlock32 sb;
    const int64_t t0 = (int64_t)blockIdx.y * DP0_TCHUNK;
    const int tcount = (int)min((int64_t)DP0_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        double c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) c[d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
        for (int p = 0; p < NQ6; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
            const float o0 = (float)(x[0] - c[0]), o1 = (float)(x[1] - c[1]), o2 = (float)(x[2] - c[2]);
            sb.o[idx][p] = make_float4(o0, o1, o2, fmaf(o2, o2, fmaf(o1, o1, o0 * o0)));
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.c[idx][d] = c[d];
            sb.n[idx][d] = (float)g.n[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        sb.ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    // trial point offsets, packed by pairs of quadrature points
    float2 yx[NP], yyy[NP], yz[NP], yy2[NP], yn2[NP], wq2[NP];
    const float sn0 = (float)gs.n[0], sn1 = (float)gs.n[1], sn2 = (float)gs.n[2];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        float o[2][3];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double v[3];
            to_global(gs, rule.x[2 * j + h], rule.y[2 * j + h], v);
#pragma unroll
            for (int d = 0; d < 3; ++d) o[h][d] = (float)(v[d] - sc[d]);
        }
        yx[j] = f2(o[0][0], o[1][0]);
        yyy[j] = f2(o[0][1], o[1][1]);
        yz[j] = f2(o[0][2], o[1][2]);
        yy2[j] = fma2(yz[j], yz[j], fma2(yyy[j], yyy[j], mul2(yx[j], yx[j])));
        yn2[j] = fma2(yz[j], b2(sn2), fma2(yyy[j], b2(sn1), mul2(yx[j], b2(sn0))));
        wq2[j] = f2(rule.wf[2 * j], rule.wf[2 * j + 1]);
    }
    const double kr = prm.p[0];
    const float2 k2 = b2((float)kr);
    const float etar_s = (float)prm.p[2], etai_s = (float)prm.p[3];

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        const bool adj = prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2);
        double acc_re = 0.0, acc_im = 0.0;
        if (!adj) {
            const double D0 = sc[0] - sb.c[tt][0], D1 = sc[1] - sb.c[tt][1], D2 = sc[2] - sb.c[tt][2];
            const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
            const double rc = sqrt(rc2);
            double ph_s = 0.0, ph_c = 1.0;
            if (T::helm) sincos_cw64(kr * rc, &ph_s, &ph_c);
            const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
            const float2 rcf2 = b2((float)rc), rc2f2 = b2((float)rc2);
            float nx0 = sn0, nx1 = sn1, nx2 = sn2;
            float2 ynq[NP];
            if (T::adjoint) {
                nx0 = sb.n[tt][0];
                nx1 = sb.n[tt][1];
                nx2 = sb.n[tt][2];
#pragma unroll
                for (int j = 0; j < NP; ++j)
                    ynq[j] = mul2(b2(-1.f), fma2(yz[j], b2(nx2), fma2(yyy[j], b2(nx1), mul2(yx[j], b2(nx0)))));
            } else {
#pragma unroll
                for (int j = 0; j < NP; ++j) ynq[j] = yn2[j];
            }
            const float Dn = fmaf(D2f, nx2, fmaf(D1f, nx1, D0f * nx0));
            const float2 D0d = b2(2.f * D0f), D1d = b2(2.f * D1f), D2d = b2(2.f * D2f);
            float2 A[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) A[j] = fma2(D2d, yz[j], fma2(D1d, yyy[j], fma2(D0d, yx[j], yy2[j])));
            double a64r = 0.0, a64i = 0.0;
            for (int p = 0; p < NQ6; ++p) {
                const float4 o = sb.o[tt][p];
                const float Bp = fmaf(-2.f, fmaf(D2f, o.z, fmaf(D1f, o.y, D0f * o.x)), o.w);
                const float cp = Dn - fmaf(o.z, nx2, fmaf(o.y, nx1, o.x * nx0));
                const float2 ox = b2(-2.f * o.x), oy = b2(-2.f * o.y), oz = b2(-2.f * o.z), Bp2 = b2(Bp);
                const float2 cp2 = b2(T::adjoint ? -cp : cp);
                // s0 = sum f e^{i theta} (single-layer part), s1 = sum f v (i k - 1/r) e^{i theta}
                float2 s0r = b2(0.f), s0i = b2(0.f), s1r = b2(0.f), s1i = b2(0.f);
#pragma unroll
                for (int j = 0; j < NP; ++j) {
                    // r^2 - r_c^2 = A_q + B_p - 2 yo_q . o_p
                    const float2 sdot = fma2(yz[j], oz, fma2(yyy[j], oy, fma2(yx[j], ox, add2(A[j], Bp2))));
                    const float2 r2 = add2(rc2f2, sdot);
                    const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    const float2 den = fma2(r2, rinv, rcf2);
                    const float2 delta = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                    const float2 f = mul2(wq2[j], rinv);
                    float2 dotv = b2(0.f);
                    if (T::normal) dotv = add2(cp2, ynq[j]);  // adjoint sign folded into cp2 / ynq
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        s0r = add2(f, s0r);
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        s1r = fma2(mul2(f, dotv), mul2(rinv, rinv), s1r);
                    } else {
                        float2 sn, cs;
                        sincos2<PHC>(mul2(k2, delta), &sn, &cs);
                        if (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                            s0r = fma2(f, cs, s0r);
                            s0i = fma2(f, sn, s0i);
                        }
                        if (K != BEMPPCUDA_HELMHOLTZ_SLP) {
                            const float2 g = mul2(f, mul2(dotv, rinv));
                            const float2 h1 = fma2(rinv, cs, mul2(k2, sn));
                            const float2 h2 = fma2(k2, cs, mul2(rinv, mul2(sn, b2(-1.f))));
                            s1r = fma2(g, h1, s1r);  // sign of -g h1 applied per test point
                            s1i = fma2(g, h2, s1i);
                        }
                    }
                }
                // combine: eta * s0 - s1r + i s1i  (Laplace DLP: -s1r; SLP: s0)
                float sr, sim;
                {
                    const float a0 = s0r.x + s0r.y, b0 = s0i.x + s0i.y, a1 = s1r.x + s1r.y, b1 = s1i.x + s1i.y;
                    if (K == BEMPPCUDA_LAPLACE_SLP || K == BEMPPCUDA_HELMHOLTZ_SLP) {
                        sr = a0;
                        sim = b0;
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        sr = -a1;
                        sim = 0.f;
                    } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                        sr = fmaf(etar_s, a0, fmaf(-etai_s, b0, -a1));
                        sim = fmaf(etar_s, b0, fmaf(etai_s, a0, b1));
                    } else {
                        sr = -a1;
                        sim = b1;
                    }
                }
                a64r = fma(rule.w[p], (double)sr, a64r);
                a64i = fma(rule.w[p], (double)sim, a64i);
            }
            const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
            acc_re = (a64r * ph_c - a64i * ph_s) * scale;
            acc_im = (a64r * ph_s + a64i * ph_c) * scale;
        }
        store_entry(prm, row, si, adj, acc_re, acc_im);
    }
}

// --------------------------------------------------------------------------------------------
// Generic element-pair kernel
// --------------------------------------------------------------------------------------------
constexpr int GEN_THREADS = 128;
constexpr int GEN_TCHUNK = 16;

__device__ __forceinline__ void atomic_add_out(void *result, int is_complex, int64_t ld, int64_t row, int64_t col,
                                               double re, double im) {
    if (is_complex) {
        double *o = reinterpret_cast<double *>(result) + 2 * (row * ld + col);
        atomicAdd(o, re);
        atomicAdd(o + 1, im);
    } else {
        atomicAdd(reinterpret_cast<double *>(result) + row * ld + col, re);
    }
}

template <int ASM, int K>
__global__ void __launch_bounds__(GEN_THREADS) regular_generic(RegParams prm, QuadRule rule) {
    __shared__ double s_x[GEN_TCHUNK][BEMPPCUDA_MAX_REGULAR_POINTS][3];
    __shared__ double s_n[GEN_TCHUNK][3];
    __shared__ double s_ie[GEN_TCHUNK];
    __shared__ int s_v[GEN_TCHUNK][3];

    const int nq = rule.nq;
    const int64_t t0 = (int64_t)blockIdx.y * GEN_TCHUNK;
    const int tcount = (int)min((int64_t)GEN_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        for (int p = 0; p < nq; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
#pragma unroll
            for (int d = 0; d < 3; ++d) s_x[idx][p][d] = x[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s_n[idx][d] = g.n[d];
            s_v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        s_ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * GEN_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    const int nt = prm.tnshape, ns = prm.snshape;
    const double kr = prm.p[0], ki = prm.p[1];
    constexpr bool HYP = (ASM == BEMPPCUDA_ASM_LAPLACE_HYP || ASM == BEMPPCUDA_ASM_HELM_HYP ||
                          ASM == BEMPPCUDA_ASM_MODHELM_HYP);
    constexpr bool MAXWELL = (ASM == BEMPPCUDA_ASM_EFIE || ASM == BEMPPCUDA_ASM_MFIE);
    double curl_s[3][3];
    if (HYP) surface_curls(prm.sg, prm.sne, s, gs.n, curl_s);
    double el_s[3] = {1.0, 1.0, 1.0};
    if (MAXWELL)
        for (int j = 0; j < 3; ++j) el_s[j] = edge_length(prm.sg, prm.sne, s, j);

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t t = prm.tsup[t0 + tt];
        if (prm.grids_identical) {
            const int a0 = s_v[tt][0], a1 = s_v[tt][1], a2 = s_v[tt][2];
            if ((a0 == sv0) | (a0 == sv1) | (a0 == sv2) | (a1 == sv0) | (a1 == sv1) | (a1 == sv2) | (a2 == sv0) |
                (a2 == sv1) | (a2 == sv2))
                continue;
        }
        const double tn[3] = {s_n[tt][0], s_n[tt][1], s_n[tt][2]};
        double lre[3][3], lim[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) lre[i][j] = lim[i][j] = 0.0;

        Geom gt;  // test geometry for the Piola transform / curls
        double curl_t[3][3];
        if (HYP || MAXWELL) {
            load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
            if (HYP) surface_curls(prm.tg, prm.tne, t, gt.n, curl_t);
        }
        const double normal_prod = tn[0] * gs.n[0] + tn[1] * gs.n[1] + tn[2] * gs.n[2];
        double cp[3][3];
        if (HYP) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    cp[i][j] = curl_t[i][0] * curl_s[j][0] + curl_t[i][1] * curl_s[j][1] + curl_t[i][2] * curl_s[j][2];
        }
        for (int p = 0; p < nq; ++p) {
            const double xp[3] = {s_x[tt][p][0], s_x[tt][p][1], s_x[tt][p][2]};
            double phi_t[3];
            scalar_shape(nt, rule.x[p], rule.y[p], phi_t);
            double bt[3][3];
            if (MAXWELL) rwg_values(gt, rule.x[p], rule.y[p], bt);
            for (int q = 0; q < nq; ++q) {
                double yq[3];
                to_global(gs, rule.x[q], rule.y[q], yq);
                const cplx kv = greens<K>(xp, yq, tn, gs.n, prm.p);
                const double wf = rule.w[p] * rule.w[q];
                const cplx tmp = cscale(kv, wf);
                double phi_s[3];
                scalar_shape(ns, rule.x[q], rule.y[q], phi_s);
                if (ASM == BEMPPCUDA_ASM_SCALAR) {
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            if (i < nt && j < ns) {
                                const double f = phi_t[i] * phi_s[j];
                                lre[i][j] = fma(tmp.re, f, lre[i][j]);
                                lim[i][j] = fma(tmp.im, f, lim[i][j]);
                            }
                        }
                } else if (HYP) {
                    // curl.curl - k^2 phi psi n.n (Helmholtz), + k^2 (modified), curl.curl (Laplace)
                    double k2r = 0.0, k2i = 0.0;
                    if (ASM == BEMPPCUDA_ASM_HELM_HYP) {
                        k2r = -(kr * kr - ki * ki);
                        k2i = -(2.0 * kr * ki);
                    } else if (ASM == BEMPPCUDA_ASM_MODHELM_HYP) {
                        k2r = kr * kr;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            const double m = phi_t[i] * phi_s[j] * normal_prod;
                            const cplx fac = {cp[i][j] + k2r * m, k2i * m};
                            const cplx v = cmul(tmp, fac);
                            lre[i][j] += v.re;
                            lim[i][j] += v.im;
                        }
                } else {
                    double bs[3][3];
                    rwg_values(gs, rule.x[q], rule.y[q], bs);
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
                        // -i k b_t.b_s - 4 / (i k |J_t| |J_s|)
                        const double div = 4.0 / (gt.ie * gs.ie);
                        // 1 / (i k) = -i conj(k) / |k|^2
                        const double kk = kr * kr + ki * ki;
                        const cplx inv_ik = {-ki / kk, -kr / kk};
                        const cplx mik = {ki, -kr};  // -i k
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) {
                                const double dot = bt[i][0] * bs[j][0] + bt[i][1] * bs[j][1] + bt[i][2] * bs[j][2];
                                const cplx fac = {mik.re * dot - div * inv_ik.re, mik.im * dot - div * inv_ik.im};
                                const cplx v = cmul(tmp, fac);
                                lre[i][j] += v.re;
                                lim[i][j] += v.im;
                            }
                    } else {
                        const double df[3] = {xp[0] - yq[0], xp[1] - yq[1], xp[2] - yq[2]};
                        const double dist2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
                        const double dist = sqrt(dist2);
                        // (i k dist - 1) / dist^2
                        const cplx f = {(-ki * dist - 1.0) / dist2, kr * dist / dist2};
                        const cplx tf = cmul(tmp, f);
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) {
                                const double c0 = bt[i][1] * bs[j][2] - bt[i][2] * bs[j][1];
                                const double c1 = bt[i][2] * bs[j][0] - bt[i][0] * bs[j][2];
                                const double c2 = bt[i][0] * bs[j][1] - bt[i][1] * bs[j][0];
                                const double tr = df[0] * c0 + df[1] * c1 + df[2] * c2;
                                lre[i][j] += tf.re * tr;
                                lim[i][j] += tf.im * tr;
                            }
                    }
                }
            }
        }
        const double scale = s_ie[tt] * gs.ie;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i >= nt) continue;
            const double mt = prm.tmult[t * nt + i];
            if (mt == 0.0) continue;
            const int64_t row = prm.tl2g[t * nt + i];
            const double elt = MAXWELL ? edge_length(prm.tg, prm.tne, t, i) : 1.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                if (j >= ns) continue;
                const double ms = prm.smult[s * ns + j];
                if (ms == 0.0) continue;
                const int64_t col = prm.sl2g[s * ns + j];
                const double f = scale * mt * ms * elt * el_s[j];
                atomic_add_out(prm.result, prm.is_complex, prm.ld, row, col, lre[i][j] * f, lim[i][j] * f);
            }
        }
    }
}

template <int K>
static cudaError_t launch_dp0(const RegParams &prm, const QuadRule &rule, int mixed, int phase_class,
                              cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS), (unsigned)((prm.ntest + DP0_TCHUNK - 1) / DP0_TCHUNK));
    const bool ck = prm.p[1] != 0.0 && KernelTraits<K>::helm;
    if constexpr (!KernelTraits<K>::modhelm) {
        if (mixed && !ck) {
            if (phase_class == 2)
                regular_dp0_mixed2<K, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            else if (phase_class == 1)
                regular_dp0_mixed2<K, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            else
                regular_dp0_mixed2<K, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            return cudaGetLastError();
        }
    }
    if (mixed) {
        if (ck)
            regular_dp0_mixed<K, true, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_dp0_mixed<K, false, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_dp0_mixed<K, false, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_dp0_mixed<K, false, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    } else {
        if (ck)
            regular_dp0_fp64<K, true, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_dp0_fp64<K, false, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_dp0_fp64<K, false, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_dp0_fp64<K, false, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    }
    return cudaGetLastError();
}

template <int ASM, int K>
static cudaError_t launch_generic(const RegParams &prm, const QuadRule &rule, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + GEN_THREADS - 1) / GEN_THREADS), (unsigned)((prm.ntest + GEN_TCHUNK - 1) / GEN_TCHUNK));
    regular_generic<ASM, K><<<grid, GEN_THREADS, 0, st>>>(prm, rule);
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

// Host entry: validated arguments in, kernel launches out.  Returns a status.
int bc_regular_launch(const bemppcuda_regular_args *a, cudaStream_t st) {
    RegParams prm;
    prm.tg = a->test_grid.geom;
    prm.sg = a->trial_grid.geom;
    prm.tne = a->test_grid.nelements;
    prm.sne = a->trial_grid.nelements;
    prm.tel = a->test_grid.elements;
    prm.sel = a->trial_grid.elements;
    prm.tsup = a->test.support;
    prm.ssup = a->trial.support;
    prm.ntest = a->test.nsupport;
    prm.ntrial = a->trial.nsupport;
    prm.tl2g = a->test.l2g;
    prm.sl2g = a->trial.l2g;
    prm.tmult = a->test.mult;
    prm.smult = a->trial.mult;
    prm.tnm = a->test.normal_mult;
    prm.snm = a->trial.normal_mult;
    prm.tnshape = a->test.nshape;
    prm.snshape = a->trial.nshape;
    prm.grids_identical = a->grids_identical;
    prm.is_complex = a->is_complex;
    prm.overwrite = a->overwrite;
    prm.pad = 0;
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    prm.result = a->result;
    prm.ld = a->ld;
    if (prm.ntest == 0 || prm.ntrial == 0) return BEMPPCUDA_OK;

    QuadRule rule;
    rule.nq = a->nq;
    rule.pad = 0;
    for (int i = 0; i < BEMPPCUDA_MAX_REGULAR_POINTS; ++i) {
        rule.x[i] = i < a->nq ? a->quad_points[2 * i] : 0.0;
        rule.y[i] = i < a->nq ? a->quad_points[2 * i + 1] : 0.0;
        rule.w[i] = i < a->nq ? a->quad_weights[i] : 0.0;
        rule.wf[i] = (float)rule.w[i];
    }

    const bool dp0 = a->assembly == BEMPPCUDA_ASM_SCALAR && a->test.nshape == 1 && a->trial.nshape == 1 &&
                     a->test.dof_is_position && a->trial.dof_is_position && a->nq == NQ6 &&
                     (a->kernel <= BEMPPCUDA_MODHELM_ADLP || a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED);
    if (a->overwrite && !dp0) {
        bc_set_error("overwrite mode needs the DP0 fast path (DP0 spaces, identity dofs, 6-point rule)");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->precision == BEMPPCUDA_MIXED && !dp0) {
        bc_set_error("mixed precision is implemented for DP0 scalar assembly with the 6-point rule");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    cudaError_t err = cudaSuccess;
    const int mixed = a->precision == BEMPPCUDA_MIXED;
    // the phase k (r - r_c) is bounded by |k| (R_test + R_trial): at most 1 or
    // 1/2 lets the sine / cosine skip the range reduction (classes 1, 2)
    const double theta = fabs(a->params[0]) * a->phase_radius;
    const int phase_class = a->phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
    if (dp0) {
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: err = launch_dp0<BEMPPCUDA_LAPLACE_SLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_LAPLACE_DLP: err = launch_dp0<BEMPPCUDA_LAPLACE_DLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_LAPLACE_ADLP: err = launch_dp0<BEMPPCUDA_LAPLACE_ADLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_MODHELM_SLP: err = launch_dp0<BEMPPCUDA_MODHELM_SLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_MODHELM_DLP: err = launch_dp0<BEMPPCUDA_MODHELM_DLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_MODHELM_ADLP: err = launch_dp0<BEMPPCUDA_MODHELM_ADLP>(prm, rule, mixed, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, mixed, phase_class, st); break;
        default: bc_set_error("kernel %d not valid for boundary assembly", a->kernel); return BEMPPCUDA_ERR_INVALID;
        }
    } else {
        switch (a->assembly) {
        case BEMPPCUDA_ASM_SCALAR:
            switch (a->kernel) {
            case BEMPPCUDA_LAPLACE_SLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_SLP>(prm, rule, st); break;
            case BEMPPCUDA_LAPLACE_DLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_DLP>(prm, rule, st); break;
            case BEMPPCUDA_LAPLACE_ADLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_SLP: err = launch_generic<0, BEMPPCUDA_MODHELM_SLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_DLP: err = launch_generic<0, BEMPPCUDA_MODHELM_DLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_ADLP: err = launch_generic<0, BEMPPCUDA_MODHELM_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, st); break;
            default: bc_set_error("kernel %d not valid for boundary assembly", a->kernel); return BEMPPCUDA_ERR_INVALID;
            }
            break;
        case BEMPPCUDA_ASM_LAPLACE_HYP: err = launch_generic<1, BEMPPCUDA_LAPLACE_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_HELM_HYP: err = launch_generic<2, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_MODHELM_HYP: err = launch_generic<3, BEMPPCUDA_MODHELM_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_EFIE: err = launch_generic<4, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_MFIE: err = launch_generic<5, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        default: bc_set_error("assembly type %d unknown", a->assembly); return BEMPPCUDA_ERR_INVALID;
        }
    }
    if (err != cudaSuccess) {
        bc_set_error("regular assembly launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
