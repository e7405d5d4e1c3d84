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
template <int K, bool MIXED>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0(RegParams prm, QuadRule rule) {
    __shared__ double s_x[DP0_TCHUNK][NQ6][3];  // test quadrature points (FP64 path) / offsets (mixed)
    __shared__ double s_n[DP0_TCHUNK][3];        // test normals
    __shared__ double s_c[DP0_TCHUNK][3];        // test centroids (mixed)
    __shared__ double s_ie[DP0_TCHUNK];
    __shared__ int s_v[DP0_TCHUNK][3];

    const int64_t t0 = (int64_t)blockIdx.y * DP0_TCHUNK;
    const int tcount = (int)min((int64_t)DP0_TCHUNK, prm.ntest - t0);

    // stage the test block
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        const double nm = prm.tnm ? (double)prm.tnm[t] : 1.0;
        load_geom(prm.tg, prm.tne, t, nm, g);
        double c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) c[d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
        for (int p = 0; p < NQ6; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
#pragma unroll
            for (int d = 0; d < 3; ++d) s_x[idx][p][d] = MIXED ? (x[d] - c[d]) : x[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s_n[idx][d] = g.n[d];
            s_c[idx][d] = c[d];
            s_v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        s_ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];

    Geom gs;
    const double snm = prm.snm ? (double)prm.snm[s] : 1.0;
    load_geom(prm.sg, prm.sne, s, snm, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);

    // trial quadrature points (absolute in FP64, centroid offsets in FP32)
    double y[NQ6][3];
    float yo[NQ6][3];
#pragma unroll
    for (int q = 0; q < NQ6; ++q) {
        double v[3];
        to_global(gs, rule.x[q], rule.y[q], v);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (MIXED)
                yo[q][d] = (float)(v[d] - sc[d]);
            else
                y[q][d] = v[d];
        }
    }
    float wqf[NQ6];
#pragma unroll
    for (int q = 0; q < NQ6; ++q) wqf[q] = (float)rule.w[q];

    const double kr = prm.p[0], ki = prm.p[1];
    const bool cplx_out = prm.is_complex;

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        bool adj = false;
        if (prm.grids_identical) {
            const int a0 = s_v[tt][0], a1 = s_v[tt][1], a2 = s_v[tt][2];
            adj = (a0 == sv0) | (a0 == sv1) | (a0 == sv2) | (a1 == sv0) | (a1 == sv1) | (a1 == sv2) |
                  (a2 == sv0) | (a2 == sv1) | (a2 == sv2);
        }
        double acc_re = 0.0, acc_im = 0.0;
        if (!adj) {
            const double tn0 = s_n[tt][0], tn1 = s_n[tt][1], tn2 = s_n[tt][2];
            if (!MIXED) {
                for (int p = 0; p < NQ6; ++p) {
                    const double x0 = s_x[tt][p][0], x1 = s_x[tt][p][1], x2 = s_x[tt][p][2];
                    double sr = 0.0, sim = 0.0;
#pragma unroll
                    for (int q = 0; q < NQ6; ++q) {
                        const double d0 = y[q][0] - x0, d1 = y[q][1] - x1, d2 = y[q][2] - x2;
                        const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                        const double rinv = rsqrt(r2);
                        if (K == BEMPPCUDA_LAPLACE_SLP) {
                            sr = fma(rule.w[q], rinv, sr);
                        } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                            double dot = (K == BEMPPCUDA_LAPLACE_DLP) ? fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]))
                                                                      : -fma(d2, tn2, fma(d1, tn1, d0 * tn0));
                            // DLP: -(y-x).n_y / r^3 ; ADLP: (y-x).n_x / r^3
                            sr = fma(-rule.w[q] * dot, rinv * rinv * rinv, sr);
                        } else if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
                            const double r = r2 * rinv;
                            double sn, cs;
                            sincos(kr * r, &sn, &cs);
                            double f = rule.w[q] * rinv;
                            if (ki != 0.0) f *= exp(-ki * r);
                            sr = fma(cs, f, sr);
                            sim = fma(sn, f, sim);
                        } else if (K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP) {
                            const double r = r2 * rinv;
                            double dot = (K == BEMPPCUDA_HELMHOLTZ_DLP) ? fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]))
                                                                        : -fma(d2, tn2, fma(d1, tn1, d0 * tn0));
                            double lg = rule.w[q] * dot * rinv * rinv * rinv;
                            if (ki != 0.0) lg *= exp(-ki * r);
                            double sn, cs;
                            sincos(kr * r, &sn, &cs);
                            const double fr = cs * lg, fi = sn * lg;
                            const double a = -1.0 - ki * r, b = kr * r;
                            sr += a * fr - b * fi;
                            sim += b * fr + a * fi;
                        } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                            // DLP + eta SLP sharing r and exp(i k r)
                            const double r = r2 * rinv;
                            const double dot = fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]));
                            double sn, cs;
                            sincos(kr * r, &sn, &cs);
                            double f = rule.w[q] * rinv;
                            if (ki != 0.0) f *= exp(-ki * r);
                            const double g = dot * rinv * rinv;
                            const double ar = fma(-1.0 - ki * r, g, prm.p[2]), ai = fma(kr * r, g, prm.p[3]);
                            const double er = cs * f, ei = sn * f;
                            sr += er * ar - ei * ai;
                            sim += er * ai + ei * ar;
                        } else if (K == BEMPPCUDA_MODHELM_SLP) {
                            const double r = r2 * rinv;
                            sr = fma(rule.w[q] * exp(-kr * r), rinv, sr);
                        } else if (K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_MODHELM_ADLP) {
                            const double r = r2 * rinv;
                            double dot = (K == BEMPPCUDA_MODHELM_DLP) ? fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]))
                                                                      : -fma(d2, tn2, fma(d1, tn1, d0 * tn0));
                            // DLP: (y-x).n_y (-k r - 1); ADLP: (y-x).n_x (k r + 1) = -(x... ) handled by sign of dot
                            sr = fma(rule.w[q] * dot * (-kr * r - 1.0) * exp(-kr * r), rinv * rinv * rinv, sr);
                        }
                    }
                    acc_re = fma(rule.w[p], sr, acc_re);
                    acc_im = fma(rule.w[p], sim, acc_im);
                }
            } else {
                // mixed precision: FP64 centroid geometry, FP32 point offsets
                const double D0 = sc[0] - s_c[tt][0], D1 = sc[1] - s_c[tt][1], D2 = sc[2] - s_c[tt][2];
                const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
                const double rc = sqrt(rc2);
                double ph_s = 0.0, ph_c = 1.0, damp = 1.0;
                if (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
                    K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                    sincos(kr * rc, &ph_s, &ph_c);
                    if (ki != 0.0) damp = exp(-ki * rc);
                } else if (K >= BEMPPCUDA_MODHELM_SLP && K <= BEMPPCUDA_MODHELM_ADLP) {
                    damp = exp(-kr * rc);
                }
                const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
                const float rcf = (float)rc, rc2f = (float)rc2;
                const float krf = (float)kr, kif = (float)ki;
                const float etar = (float)prm.p[2], etai = (float)prm.p[3];
                const float tn0f = (float)tn0, tn1f = (float)tn1, tn2f = (float)tn2;
                const float sn0f = (float)gs.n[0], sn1f = (float)gs.n[1], sn2f = (float)gs.n[2];
                double a64r = 0.0, a64i = 0.0;
                for (int p = 0; p < NQ6; ++p) {
                    const float o0 = (float)s_x[tt][p][0], o1 = (float)s_x[tt][p][1], o2 = (float)s_x[tt][p][2];
                    float sr = 0.f, sim = 0.f;
#pragma unroll
                    for (int q = 0; q < NQ6; ++q) {
                        // e = (y_q - c_s) - (x_p - c_t); d = y - x = D + e
                        const float e0 = yo[q][0] - o0, e1 = yo[q][1] - o1, e2 = yo[q][2] - o2;
                        const float sdot = fmaf(e2, fmaf(2.f, D2f, e2), fmaf(e1, fmaf(2.f, D1f, e1), e0 * fmaf(2.f, D0f, e0)));
                        const float r2 = rc2f + sdot;
                        const float rinv = rsqrtf(r2);
                        const float r = r2 * rinv;
                        const float delta = __fdividef(sdot, r + rcf);
                        const float d0 = D0f + e0, d1 = D1f + e1, d2 = D2f + e2;
                        if (K == BEMPPCUDA_LAPLACE_SLP) {
                            sr = fmaf(wqf[q], rinv, sr);
                        } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                            float dot = (K == BEMPPCUDA_LAPLACE_DLP) ? fmaf(d2, sn2f, fmaf(d1, sn1f, d0 * sn0f))
                                                                     : -fmaf(d2, tn2f, fmaf(d1, tn1f, d0 * tn0f));
                            sr = fmaf(-wqf[q] * dot, rinv * rinv * rinv, sr);
                        } else if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
                            float sn, cs;
                            sincosf(krf * delta, &sn, &cs);
                            float f = wqf[q] * rinv;
                            if (kif != 0.f) f *= expf(-kif * delta);
                            sr = fmaf(cs, f, sr);
                            sim = fmaf(sn, f, sim);
                        } else if (K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP) {
                            float dot = (K == BEMPPCUDA_HELMHOLTZ_DLP) ? fmaf(d2, sn2f, fmaf(d1, sn1f, d0 * sn0f))
                                                                       : -fmaf(d2, tn2f, fmaf(d1, tn1f, d0 * tn0f));
                            float lg = wqf[q] * dot * rinv * rinv * rinv;
                            if (kif != 0.f) lg *= expf(-kif * delta);
                            float sn, cs;
                            sincosf(krf * delta, &sn, &cs);
                            const float fr = cs * lg, fi = sn * lg;
                            const float a = -1.f - kif * r, b = krf * r;
                            sr += a * fr - b * fi;
                            sim += b * fr + a * fi;
                        } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                            const float dot = fmaf(d2, sn2f, fmaf(d1, sn1f, d0 * sn0f));
                            float sn, cs;
                            sincosf(krf * delta, &sn, &cs);
                            float f = wqf[q] * rinv;
                            if (kif != 0.f) f *= expf(-kif * delta);
                            const float g = dot * rinv * rinv;
                            const float ar = fmaf(-1.f - kif * r, g, etar), ai = fmaf(krf * r, g, etai);
                            const float er = cs * f, ei = sn * f;
                            sr += er * ar - ei * ai;
                            sim += er * ai + ei * ar;
                        } else if (K == BEMPPCUDA_MODHELM_SLP) {
                            sr = fmaf(wqf[q] * expf(-krf * delta), rinv, sr);
                        } else if (K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_MODHELM_ADLP) {
                            float dot = (K == BEMPPCUDA_MODHELM_DLP) ? fmaf(d2, sn2f, fmaf(d1, sn1f, d0 * sn0f))
                                                                     : -fmaf(d2, tn2f, fmaf(d1, tn1f, d0 * tn0f));
                            sr = fmaf(wqf[q] * dot * (-krf * r - 1.f) * expf(-krf * delta), rinv * rinv * rinv, sr);
                        }
                    }
                    a64r = fma(rule.w[p], (double)sr, a64r);
                    a64i = fma(rule.w[p], (double)sim, a64i);
                }
                // multiply by exp(i k r_c) (and the damping of Im k / modified Helmholtz)
                a64r *= damp;
                a64i *= damp;
                acc_re = a64r * ph_c - a64i * ph_s;
                acc_im = a64r * ph_s + a64i * ph_c;
            }
            const double scale = BC_INV_4PI * s_ie[tt] * gs.ie;
            acc_re *= scale;
            acc_im *= scale;
        }
        if (cplx_out) {
            double2 *out = reinterpret_cast<double2 *>(prm.result) + row * prm.ld + si;
            if (prm.overwrite) {
                *out = make_double2(acc_re, acc_im);
            } else if (!adj) {
                double2 old = *out;
                *out = make_double2(old.x + acc_re, old.y + acc_im);
            }
        } else {
            double *out = reinterpret_cast<double *>(prm.result) + row * prm.ld + si;
            if (prm.overwrite)
                *out = acc_re;
            else if (!adj)
                *out += acc_re;
        }
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
static cudaError_t launch_dp0(const RegParams &prm, const QuadRule &rule, int mixed, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS), (unsigned)((prm.ntest + DP0_TCHUNK - 1) / DP0_TCHUNK));
    if (mixed)
        regular_dp0<K, true><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    else
        regular_dp0<K, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
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
    if (dp0) {
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: err = launch_dp0<BEMPPCUDA_LAPLACE_SLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_LAPLACE_DLP: err = launch_dp0<BEMPPCUDA_LAPLACE_DLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_LAPLACE_ADLP: err = launch_dp0<BEMPPCUDA_LAPLACE_ADLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_MODHELM_SLP: err = launch_dp0<BEMPPCUDA_MODHELM_SLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_MODHELM_DLP: err = launch_dp0<BEMPPCUDA_MODHELM_DLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_MODHELM_ADLP: err = launch_dp0<BEMPPCUDA_MODHELM_ADLP>(prm, rule, mixed, st); break;
        case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, mixed, st); break;
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
