// DP0 regular-pair tiles shared by the single-problem kernels (regular.cu)
// and the persistent multi-problem kernel (batch.cu).  One tile is a block of
// up to DP0_TCHUNK test elements (rows) x DP0_THREADS trial elements (columns).
#pragma once

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
    int defer_transpose;  // symmetric P1 sweep into a zeroed result: skip the (j, i) blocks (added later as U^T)
    double p[4];
    void *result;
    int64_t ld;
    double near_r;  // bound on the centroid distance of vertex-sharing pairs (0: unknown, test every pair)
    void *tresult;  // stripe mode of the symmetric DP0 sweeps (store_pair): transposed entries, local rows
    int64_t row0, col0;
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

// Both entries of a symmetric-sweep pair (row i <= column j): A_ij at (i, j) and A_ji at (j, i) of the
// matrix, or in stripe mode (STRIPE, prm.tresult set) A_ij at (i - row0, j - col0) of result and A_ji
// at the same position of tresult, so both stores of a warp are coalesced.  A template switch, so the
// single-GPU sweeps carry no stripe branch.
template <bool STRIPE>
__device__ __forceinline__ void store_pair(const RegParams &prm, int64_t row, int64_t col, bool adj, double a_re,
                                           double a_im, double b_re, double b_im) {
    if (STRIPE) {
        const int64_t at = (row - prm.row0) * prm.ld + (col - prm.col0);
        if (prm.is_complex) {
            double2 *o = reinterpret_cast<double2 *>(prm.result) + at;
            double2 *ot = reinterpret_cast<double2 *>(prm.tresult) + at;
            if (prm.overwrite) {
                *o = make_double2(a_re, a_im);
                if (row != col) *ot = make_double2(b_re, b_im);
            } else if (!adj) {
                const double2 u = *o;
                *o = make_double2(u.x + a_re, u.y + a_im);
                if (row != col) {
                    const double2 v = *ot;
                    *ot = make_double2(v.x + b_re, v.y + b_im);
                }
            }
        } else {
            double *o = reinterpret_cast<double *>(prm.result) + at;
            double *ot = reinterpret_cast<double *>(prm.tresult) + at;
            if (prm.overwrite) {
                *o = a_re;
                if (row != col) *ot = b_re;
            } else if (!adj) {
                *o += a_re;
                if (row != col) *ot += b_re;
            }
        }
        return;
    }
    store_entry(prm, row, col, adj, a_re, a_im);
    if (row != col) store_entry(prm, col, row, adj, b_re, b_im);
}

// FP64: one thread per (trial element, block of 32 test elements).
// CK: the wavenumber has a nonzero imaginary part.
// PHC > 0: |k| (R_t + R_s) <= 1 (class 1) or <= 1/2 (class 2), so
// exp(i k r) = exp(i k r_c) exp(i k (r - r_c)) with r_c the centroid
// distance: the first factor once per element pair, the second from a
// polynomial without range reduction (r - r_c is exact to ~1e-16 r in FP64,
// so no cancellation concern here).  PHC = 0 reduces every argument.
template <int K, bool CK, int PHC>
__device__ __forceinline__ void regular_dp0_fp64_tile(const RegParams &prm, const QuadRule &rule,
                                                    int64_t tile_x, int64_t t0, int rows, TestBlock64 &sb) {
    using T = KernelTraits<K>;
    constexpr bool PH = PHC > 0 && T::helm && !CK;  // phase factored about the centroids
    // rows <= DP0_TCHUNK test elements starting at t0
    const int tcount = (int)min((int64_t)rows, prm.ntest - t0);
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

    const int64_t si = tile_x * DP0_THREADS + threadIdx.x;
    if (si < prm.ntrial) {
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
                    const double rinv = rsqrt64(r2);
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
    __syncthreads();  // the shared block is reused by the next tile of a persistent loop
}

template <int K, bool CK, int PHC>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_fp64(RegParams prm, QuadRule rule) {
    __shared__ TestBlock64 sb;
    regular_dp0_fp64_tile<K, CK, PHC>(prm, rule, blockIdx.x, (int64_t)blockIdx.y * DP0_TCHUNK, DP0_TCHUNK, sb);
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
__device__ __forceinline__ void regular_dp0_mixed_tile(const RegParams &prm, const QuadRule &rule,
                                                    int64_t tile_x, int64_t t0, int rows, TestBlock32 &sb) {
    using T = KernelTraits<K>;
    // rows <= DP0_TCHUNK test elements starting at t0
    const int tcount = (int)min((int64_t)rows, prm.ntest - t0);
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

    const int64_t si = tile_x * DP0_THREADS + threadIdx.x;
    if (si < prm.ntrial) {
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
    __syncthreads();  // the shared block is reused by the next tile of a persistent loop
}

template <int K, bool CK, int PHC>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_mixed(RegParams prm, QuadRule rule) {
    __shared__ TestBlock32 sb;
    regular_dp0_mixed_tile<K, CK, PHC>(prm, rule, blockIdx.x, (int64_t)blockIdx.y * DP0_TCHUNK, DP0_TCHUNK, sb);
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
        constexpr float ps[] = BC_SIN_HALF32;
        constexpr float pc[] = BC_COS_HALF32;
        const float2 x2 = mul2(x, x);
        *s = fma2(mul2(x, x2), fma2(b2(ps[0]), x2, b2(ps[1])), x);
        *c = fma2(x2, fma2(fma2(b2(pc[0]), x2, b2(pc[1])), x2, b2(pc[2])), b2(1.0f));
    } else if (PHC == 1) {
        constexpr float ps[] = BC_SIN_SMALL32;
        constexpr float pc[] = BC_COS_SMALL32;
        const float2 x2 = mul2(x, x);
        *s = fma2(mul2(x, x2), fma2(fma2(b2(ps[0]), x2, b2(ps[1])), x2, b2(ps[2])), x);
        *c = fma2(x2, fma2(fma2(fma2(b2(pc[0]), x2, b2(pc[1])), x2, b2(pc[2])), x2, b2(pc[3])), b2(1.0f));
    } else {
        sincos_cw32(x.x, &s->x, &c->x);
        sincos_cw32(x.y, &s->y, &c->y);
    }
}

// Test block of the packed path: per test point m = -2 kappa (x_p - c_t) and
// |kappa (x_p - c_t)|^2, with kappa = k (Helmholtz) or 1 (Laplace).
struct TestBlock32p {
    float4 m[DP0_TCHUNK][NQ6];
    double c[DP0_TCHUNK][3];  // centroid
    float n[DP0_TCHUNK][3];
    double ie[DP0_TCHUNK];
    int v[DP0_TCHUNK][3];
};

// Lengths are measured in units of 1/k (kappa = k > 0, Laplace kappa = 1):
// with primes for scaled quantities r' = k r, the phase offset is
// theta = r' - r_c' with no multiplication by k, and
//   e^{ikr}/r          = k e^{i theta'} / r',
//   (ikr - 1)(d.n)/r^3 = k^2 (i r' - 1)(d'.n) / r'^3,
// so per quadrature-point pair (f = w_q / r', g1 = f (d'.n) / r', g0 = g1 / r')
//   SLP part: sum f (cos, sin)
//   DLP part: (i r' - 1) g0 (cos + i sin) = -(g0 cos + g1 sin) + i (g1 cos - g0 sin),
// accumulated as four packed sums.  The FP32 sums run over the test points of
// one quadrature weight (the order-4 rule has two orbits of three points) and
// are then added in FP64 with that weight; kappa, eta and the centroid phase
// exp(i k r_c) are applied per entry in FP64.
template <int K, int PHC>
__device__ __forceinline__ void regular_dp0_mixed2_tile(const RegParams &prm, const QuadRule &rule,
                                                    int64_t tile_x, int64_t t0, int rows, TestBlock32p &sb) {
    using T = KernelTraits<K>;
    constexpr int NP = NQ6 / 2;
    constexpr bool DL = T::normal;  // double-layer type (DLP, ADLP, combined)
    const double kap = T::helm ? prm.p[0] : 1.0;  // callers guarantee k > 0 for the Helmholtz family
    // rows <= DP0_TCHUNK test elements starting at t0
    const int tcount = (int)min((int64_t)rows, prm.ntest - t0);
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
            const float o0 = (float)(kap * (x[0] - c[0])), o1 = (float)(kap * (x[1] - c[1])),
                        o2 = (float)(kap * (x[2] - c[2]));
            sb.m[idx][p] = make_float4(-2.f * o0, -2.f * o1, -2.f * o2, fmaf(o2, o2, fmaf(o1, o1, o0 * o0)));
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

    const int64_t si = tile_x * DP0_THREADS + threadIdx.x;
    if (si < prm.ntrial) {
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    // scaled trial point offsets, packed by pairs of quadrature points
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
            for (int d = 0; d < 3; ++d) o[h][d] = (float)(kap * (v[d] - sc[d]));
        }
        yx[j] = f2(o[0][0], o[1][0]);
        yyy[j] = f2(o[0][1], o[1][1]);
        yz[j] = f2(o[0][2], o[1][2]);
        yy2[j] = fma2(yz[j], yz[j], fma2(yyy[j], yyy[j], mul2(yx[j], yx[j])));
        yn2[j] = fma2(yz[j], b2(sn2), fma2(yyy[j], b2(sn1), mul2(yx[j], b2(sn0))));
        wq2[j] = f2(rule.wf[2 * j], rule.wf[2 * j + 1]);
    }
    // per-entry factors: kappa eta (SLP part; eta = 1 for a single layer), kappa^2 (DLP part)
    const double ek_r = (K == BEMPPCUDA_HELMHOLTZ_COMBINED) ? kap * prm.p[2] : kap;
    const double ek_i = (K == BEMPPCUDA_HELMHOLTZ_COMBINED) ? kap * prm.p[3] : 0.0;
    const double k2d = kap * kap;

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        const bool adj = prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2);
        double acc_re = 0.0, acc_im = 0.0;
        if (!adj) {
            const double D0 = kap * (sc[0] - sb.c[tt][0]), D1 = kap * (sc[1] - sb.c[tt][1]),
                         D2 = kap * (sc[2] - sb.c[tt][2]);
            const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
            const double rc = sqrt(rc2);
            double ph_s = 0.0, ph_c = 1.0;
            if (T::helm) sincos_cw64(rc, &ph_s, &ph_c);
            const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
            const float2 rcf2 = b2((float)rc), rc2f2 = b2((float)rc2);
            // dotv' = k (y - x).n_s (DLP) or -k (y - x).n_t (ADLP) = cp_p + ynq_q
            float nh0 = 0.f, nh1 = 0.f, nh2 = 0.f, Dn = 0.f;
            float2 ynq[NP];
            if (DL) {
                if (T::adjoint) {
                    const float nx0 = sb.n[tt][0], nx1 = sb.n[tt][1], nx2 = sb.n[tt][2];
#pragma unroll
                    for (int j = 0; j < NP; ++j)
                        ynq[j] = fma2(yz[j], b2(-nx2), fma2(yyy[j], b2(-nx1), mul2(yx[j], b2(-nx0))));
                    Dn = -fmaf(D2f, nx2, fmaf(D1f, nx1, D0f * nx0));
                    nh0 = -0.5f * nx0;
                    nh1 = -0.5f * nx1;
                    nh2 = -0.5f * nx2;
                } else {
#pragma unroll
                    for (int j = 0; j < NP; ++j) ynq[j] = yn2[j];
                    Dn = fmaf(D2f, sn2, fmaf(D1f, sn1, D0f * sn0));
                    nh0 = 0.5f * sn0;
                    nh1 = 0.5f * sn1;
                    nh2 = 0.5f * sn2;
                }
            }
            const float2 D0d = b2(2.f * D0f), D1d = b2(2.f * D1f), D2d = b2(2.f * D2f);
            float2 A[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) A[j] = fma2(D2d, yz[j], fma2(D1d, yyy[j], fma2(D0d, yx[j], yy2[j])));
            double er = 0.0, ei = 0.0;
            float2 s0r = b2(0.f), s0i = b2(0.f), P = b2(0.f), Q = b2(0.f), R = b2(0.f), S = b2(0.f);
            for (int p = 0; p < NQ6; ++p) {
                const float4 m = sb.m[tt][p];
                // r'^2 - r_c'^2 = A_q + B_p - 2 yo'_q . o'_p,  B_p = |o'_p|^2 - 2 D'.o'_p
                const float Bp = fmaf(D2f, m.z, fmaf(D1f, m.y, fmaf(D0f, m.x, m.w)));
                const float2 mx = b2(m.x), my = b2(m.y), mz = b2(m.z), Bp2 = b2(Bp);
                float2 cp2 = b2(0.f);
                if (DL) cp2 = b2(fmaf(m.z, nh2, fmaf(m.y, nh1, fmaf(m.x, nh0, Dn))));
#pragma unroll
                for (int j = 0; j < NP; ++j) {
                    const float2 sdot = fma2(yz[j], mz, fma2(yyy[j], my, fma2(yx[j], mx, add2(A[j], Bp2))));
                    const float2 r2 = add2(rc2f2, sdot);
                    const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    const float2 f = mul2(wq2[j], rinv);
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        s0r = add2(f, s0r);
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        const float2 g1 = mul2(mul2(f, add2(cp2, ynq[j])), rinv);
                        P = fma2(g1, rinv, P);
                    } else {
                        const float2 den = fma2(r2, rinv, rcf2);
                        const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                        float2 sn, cs;
                        sincos2<PHC>(th, &sn, &cs);
                        if (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                            s0r = fma2(f, cs, s0r);
                            s0i = fma2(f, sn, s0i);
                        }
                        if (DL) {
                            const float2 g1 = mul2(mul2(f, add2(cp2, ynq[j])), rinv);
                            const float2 g0 = mul2(g1, rinv);
                            P = fma2(g0, cs, P);
                            Q = fma2(g1, sn, Q);
                            R = fma2(g1, cs, R);
                            S = fma2(g0, sn, S);
                        }
                    }
                }
                // flush the FP32 sums where the test-point weight changes:
                // entry += w_p [kappa eta S0 + kappa^2 (-(P + Q) + i (R - S))]
                if (p == NQ6 - 1 || rule.w[p + 1] != rule.w[p]) {
                    const double wp = rule.w[p];
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        er = fma(wp, (double)(s0r.x + s0r.y), er);
                        s0r = b2(0.f);
                    } else if (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP) {
                        er = fma(-wp, (double)(P.x + P.y), er);
                        P = b2(0.f);
                    } else {
                        double vr = 0.0, vi = 0.0;
                        if (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
                            const double sr = (double)(s0r.x + s0r.y), sim = (double)(s0i.x + s0i.y);
                            vr = fma(ek_r, sr, -ek_i * sim);
                            vi = fma(ek_r, sim, ek_i * sr);
                            s0r = s0i = b2(0.f);
                        }
                        if (DL) {
                            const float2 pq = add2(P, Q);
                            const float2 rs = fma2(S, b2(-1.f), R);
                            vr = fma(-k2d, (double)(pq.x + pq.y), vr);
                            vi = fma(k2d, (double)(rs.x + rs.y), vi);
                            P = Q = R = S = b2(0.f);
                        }
                        er = fma(wp, vr, er);
                        ei = fma(wp, vi, ei);
                    }
                }
            }
            const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
            acc_re = (er * ph_c - ei * ph_s) * scale;
            acc_im = (er * ph_s + ei * ph_c) * scale;
        }
        store_entry(prm, row, si, adj, acc_re, acc_im);
    }
    }
    __syncthreads();  // the shared block is reused by the next tile of a persistent loop
}

// CTAs per SM the packed entrywise kernel is compiled for: 4 (128 registers,
// no spills) was 2 % faster than 5 (96 registers, small spills) at L6.
#ifndef BC_MIXED2_MIN_BLOCKS
#define BC_MIXED2_MIN_BLOCKS 4
#endif

template <int K, int PHC>
__global__ void __launch_bounds__(DP0_THREADS, BC_MIXED2_MIN_BLOCKS) regular_dp0_mixed2(RegParams prm, QuadRule rule) {
    __shared__ TestBlock32p sb;
    regular_dp0_mixed2_tile<K, PHC>(prm, rule, blockIdx.x, (int64_t)blockIdx.y * DP0_TCHUNK, DP0_TCHUNK, sb);
}

}  // namespace bc
