// Symmetric DP0 tiles: test and trial are the same DP0 space on one grid, so
// the element pair (i, j) and its transpose (j, i) use the same quadrature
// points with the roles of x and y exchanged.  One sweep over the 36 point
// pairs of (i, j), i < j, gives both entries:
//   single layer      A_ij = A_ji            (the kernel is symmetric in x, y)
//   double layer      A_ij with (y - x).n_j, A_ji with (x - y).n_i
//   adjoint double    the double-layer pair with the two entries exchanged
//   combined field    double layer + eta * the shared single layer
// so r, 1/r and exp(ikr) are evaluated once per point pair for two entries.
// A launch covers the tiles on or above the diagonal (row chunk <= column
// block); inside a diagonal tile only i <= j is processed, and i == j (the
// coincident pair, always adjacent) is zeroed for the singular pass.
// Entry (i, j) is stored by the thread of column j (coalesced); entry (j, i)
// lands in row j (one 8- or 16-byte store per row, merged in L2 with the
// stores of neighbouring rows of the same warp).
#pragma once

#include "dp0.cuh"

namespace bc {

template <int K>
struct SymTraits {
    static constexpr bool slp_part = (K == BEMPPCUDA_LAPLACE_SLP || K == BEMPPCUDA_HELMHOLTZ_SLP ||
                                      K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool dlp_part = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP ||
                                      K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
                                      K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_MODHELM_ADLP ||
                                      K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool swap = (K == BEMPPCUDA_LAPLACE_ADLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
                                  K == BEMPPCUDA_MODHELM_ADLP);
    static constexpr bool helm = KernelTraits<K>::helm;
    static constexpr bool modhelm = KernelTraits<K>::modhelm;
    static constexpr bool supported = slp_part || dlp_part;
};

struct TestBlock64s {
    double x[DP0_TCHUNK][NQ6][3];
    double c[DP0_TCHUNK][3];
    double n[DP0_TCHUNK][3];
    double ie[DP0_TCHUNK];
    int v[DP0_TCHUNK][3];
};

// FP64.  PHC 0-2 as in regular_dp0_fp64_tile (real wavenumber); PHC 3 is a complex wavenumber
// k = kr + i ki: exp(i kr r) from the reduced sine / cosine times exp(-ki r) per point pair and
// (ikr - 1) / r = -(1/r + ki) + i kr in the double layer (no centroid factoring: the amplitude
// varies over the pair).  G(x, y) = G(y, x) for complex k too, so the sweep is unchanged.
// Modified Helmholtz (real, w = p[0]): the Laplace sums with exp(-w r) (single layer) and
// exp(-w r) (1 + w r) (double layers) per point pair.
//
// The tile is split into three steps shared by the assembly (stores A_ij, A_ji) and the
// matrix-free apply (accumulates A x): staging the test block, loading a thread's trial
// element, and the sweep over the 36 point pairs of one element pair.

// Stage test elements t0 .. t0 + tcount - 1 (points, centroids, normals, areas, vertex ids).
__device__ __forceinline__ void stage_sym64(const RegParams &prm, const QuadRule &rule, int64_t t0, int tcount,
                                            TestBlock64s &sb) {
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
#pragma unroll
            for (int d = 0; d < 3; ++d) sb.x[idx][p][d] = x[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.n[idx][d] = g.n[d];
            sb.c[idx][d] = c[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        sb.ie[idx] = g.ie;
    }
}

// One thread's trial element: geometry, vertex ids, centroid (phase classes 1, 2) and points.
struct SymTrial64 {
    Geom gs;
    int sv0, sv1, sv2;
    double sc[3];
    double y[NQ6][3];
};

template <int K, int PHC>
__device__ __forceinline__ void load_trial_sym64(const RegParams &prm, const QuadRule &rule, int64_t si,
                                                 SymTrial64 &tr) {
    constexpr bool PH = (PHC == 1 || PHC == 2) && SymTraits<K>::helm;
    const int64_t s = prm.ssup[si];
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, tr.gs);
    tr.sv0 = __ldg(prm.sel + 3 * s);
    tr.sv1 = __ldg(prm.sel + 3 * s + 1);
    tr.sv2 = __ldg(prm.sel + 3 * s + 2);
#pragma unroll
    for (int d = 0; d < 3; ++d) tr.sc[d] = PH ? __ldg(prm.sg + (22 + d) * prm.sne + s) : 0.0;
#pragma unroll
    for (int q = 0; q < NQ6; ++q) to_global(tr.gs, rule.x[q], rule.y[q], tr.y[q]);
}

// A_ij and A_ji of the non-adjacent pair (test element tt of the block, the thread's trial element).
template <int K, int PHC>
__device__ __forceinline__ void pair_sym64(const RegParams &prm, const QuadRule &rule, const TestBlock64s &sb,
                                           int tt, const SymTrial64 &tr, double &a_re, double &a_im, double &b_re,
                                           double &b_im) {
    using ST = SymTraits<K>;
    constexpr bool PH = (PHC == 1 || PHC == 2) && ST::helm;
    constexpr bool CK = PHC == 3 && ST::helm;
    const Geom &gs = tr.gs;
    const double kr = prm.p[0], ki = CK ? prm.p[1] : 0.0, etar = prm.p[2], etai = prm.p[3];
    double rc = 0.0, ph_s = 0.0, ph_c = 1.0;
    if (PH) {
        const double D0 = tr.sc[0] - sb.c[tt][0], D1 = tr.sc[1] - sb.c[tt][1], D2 = tr.sc[2] - sb.c[tt][2];
        rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
        sincos_cw64(kr * rc, &ph_s, &ph_c);
    }
    // Normal terms: (y - x).n_j = (v0_j - x).n_j since y lies in the plane of j (one value per
    // test point, applied after the sum over q), and (x - y).n_i = (c_i - y).n_i since x lies in
    // the plane of i (one value per trial point)
    double ynt[NQ6];
    if (ST::dlp_part)
#pragma unroll
        for (int q = 0; q < NQ6; ++q)
            ynt[q] = fma(sb.c[tt][2] - tr.y[q][2], sb.n[tt][2],
                         fma(sb.c[tt][1] - tr.y[q][1], sb.n[tt][1], (sb.c[tt][0] - tr.y[q][0]) * sb.n[tt][0]));
    double s0r = 0.0, s0i = 0.0, u_re = 0.0, u_im = 0.0, v_re = 0.0, v_im = 0.0;
    for (int p = 0; p < NQ6; ++p) {
        const double x0 = sb.x[tt][p][0], x1 = sb.x[tt][p][1], x2 = sb.x[tt][p][2];
        double xn = 0.0;
        if (ST::dlp_part)
            xn = fma(gs.v0[2] - x2, gs.n[2], fma(gs.v0[1] - x1, gs.n[1], (gs.v0[0] - x0) * gs.n[0]));
        double pr = 0.0, pi = 0.0, ur = 0.0, ui = 0.0, vr = 0.0, vi = 0.0;
#pragma unroll
        for (int q = 0; q < NQ6; ++q) {
            const double d0 = tr.y[q][0] - x0, d1 = tr.y[q][1] - x1, d2 = tr.y[q][2] - x2;
            const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
            const double rinv = rsqrt64(r2);
            const double f = rule.w[q] * rinv;
            if (!ST::helm) {
                double e = 1.0, e1 = 1.0;  // modified Helmholtz: exp(-w r), exp(-w r) (1 + w r)
                if (ST::modhelm) {
                    const double r = r2 * rinv;
                    e = exp(-kr * r);
                    e1 = e * fma(kr, r, 1.0);
                }
                if (ST::slp_part) pr = ST::modhelm ? fma(f, e, pr) : pr + f;
                if (ST::dlp_part) {
                    const double g3 = ST::modhelm ? f * rinv * rinv * e1 : f * rinv * rinv;
                    ur += g3;
                    vr = fma(g3, ynt[q], vr);
                }
            } else {
                const double r = r2 * rinv;
                double sn, cs;
                if (PH && PHC == 2)
                    sincos_half64(kr * (r - rc), &sn, &cs);
                else if (PH)
                    sincos_small64(kr * (r - rc), &sn, &cs);
                else
                    sincos_cw64(kr * r, &sn, &cs);
                if (CK) {
                    const double am = exp(-ki * r);
                    sn *= am;
                    cs *= am;
                }
                if (ST::slp_part) {
                    pr = fma(f, cs, pr);
                    pi = fma(f, sn, pi);
                }
                if (ST::dlp_part) {
                    // (ikr - 1) e^{ikr} / r^3: -h1 + i h2 per unit f (dot) / r
                    const double fr = f * rinv, rk = CK ? rinv + ki : rinv;
                    const double h1 = fma(rk, cs, kr * sn), h2 = fma(kr, cs, -rk * sn);
                    const double gt = fr * ynt[q];
                    ur = fma(fr, h1, ur);
                    ui = fma(fr, h2, ui);
                    vr = fma(gt, h1, vr);
                    vi = fma(gt, h2, vi);
                }
            }
        }
        const double wp = rule.w[p], wpn = wp * xn;
        s0r = fma(wp, pr, s0r);
        s0i = fma(wp, pi, s0i);
        u_re = fma(wpn, ur, u_re);
        u_im = fma(wpn, ui, u_im);
        v_re = fma(wp, vr, v_re);
        v_im = fma(wp, vi, v_im);
    }
    // kernel values: Laplace DLP -sum f dot / r^2; Helmholtz DLP -u_re + i u_im
    double dr = 0.0, di = 0.0, er = 0.0, ei = 0.0;  // double-layer parts of A_ij, A_ji
    if (ST::dlp_part) {
        dr = -u_re;
        di = ST::helm ? u_im : 0.0;
        er = -v_re;
        ei = ST::helm ? v_im : 0.0;
    }
    if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
        const double sr = fma(etar, s0r, -etai * s0i), sim = fma(etar, s0i, etai * s0r);
        a_re = dr + sr;
        a_im = di + sim;
        b_re = er + sr;
        b_im = ei + sim;
    } else if (ST::slp_part) {
        a_re = b_re = s0r;
        a_im = b_im = s0i;
    } else if (ST::swap) {
        a_re = er;
        a_im = ei;
        b_re = dr;
        b_im = di;
    } else {
        a_re = dr;
        a_im = di;
        b_re = er;
        b_im = ei;
    }
    const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
    if (PH) {
        double t = a_re * ph_c - a_im * ph_s;
        a_im = (a_re * ph_s + a_im * ph_c) * scale;
        a_re = t * scale;
        t = b_re * ph_c - b_im * ph_s;
        b_im = (b_re * ph_s + b_im * ph_c) * scale;
        b_re = t * scale;
    } else {
        a_re *= scale;
        a_im *= scale;
        b_re *= scale;
        b_im *= scale;
    }
}

template <int K, int PHC, bool STRIPE = false>
__device__ __forceinline__ void regular_dp0_fp64_sym_tile(const RegParams &prm, const QuadRule &rule,
                                                        int64_t tile_x, int64_t t0, int rows, TestBlock64s &sb) {
    const int tcount = (int)min((int64_t)rows, prm.ntest - t0);
    stage_sym64(prm, rule, t0, tcount, sb);
    __syncthreads();

    const int64_t si = tile_x * DP0_THREADS + threadIdx.x;
    if (si < prm.ntrial && t0 <= si) {
        SymTrial64 tr;
        load_trial_sym64<K, PHC>(prm, rule, si, tr);
        for (int tt = 0; tt < tcount; ++tt) {
            const int64_t row = t0 + tt;
            if (row > si) break;  // rows increase with tt: the rest of this column lies below the diagonal
            const bool adj = row == si || (prm.grids_identical && shares_vertex(sb.v[tt], tr.sv0, tr.sv1, tr.sv2));
            double a_re = 0.0, a_im = 0.0, b_re = 0.0, b_im = 0.0;  // A_ij, A_ji
            if (!adj) pair_sym64<K, PHC>(prm, rule, sb, tt, tr, a_re, a_im, b_re, b_im);
            store_pair<STRIPE>(prm, row, si, adj, a_re, a_im, b_re, b_im);
        }
    }
    __syncthreads();  // the shared block is reused by the next tile of a persistent loop
}

}  // namespace bc

namespace bc {

// Test block of the packed symmetric sweep: per test point the scaled offset
// o = kappa (x_p - c_t) as -2 o, each component stored twice so that it is an
// f32x2 operand straight from shared memory, and |o|^2.
struct TestBlock32q {
    float4 mxy[DP0_TCHUNK][NQ6];  // (-2 o_x, -2 o_x, -2 o_y, -2 o_y)
    float4 mzw[DP0_TCHUNK][NQ6];  // (-2 o_z, -2 o_z, |o|^2, |o|^2)
    double c[DP0_TCHUNK][3];      // centroid
    float4 n[DP0_TCHUNK];         // unit normal (fourth entry unused)
    double ie[DP0_TCHUNK];
    int v[DP0_TCHUNK][3];
};

// sin / cos of the point-pair phase offsets of the symmetric sweep (|x| <= 1/2 for phase class
// 2, |x| <= 1 for class 1): the sine by the FP32 minimax polynomial, the cosine by the hardware
// approximation cos.approx.f32 (absolute error below 1e-6 on these ranges; the operator error of
// the sweep measured against FP64 is 1.3e-8 either way).  The cosine moves from the FMA pipe
// to the special-function unit, which this kernel leaves partly idle (its reciprocal and
// reciprocal square root are the other users); the sine stays a polynomial, since both
// functions on that unit saturate it.  Class 0 reduces the argument first (sincos2).
__device__ __forceinline__ float hw_cos(float x) {
    float y;
    asm("cos.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

template <int PHC>
__device__ __forceinline__ void sincos2_sym(float2 x, float2 *s, float2 *c) {
    if (PHC == 2 || PHC == 1) {
        const float2 x2 = mul2(x, x);
        if (PHC == 2) {
            constexpr float ps[] = BC_SIN_HALF32;
            *s = fma2(mul2(x, x2), fma2(b2(ps[0]), x2, b2(ps[1])), x);
        } else {
            constexpr float ps[] = BC_SIN_SMALL32;
            *s = fma2(mul2(x, x2), fma2(fma2(b2(ps[0]), x2, b2(ps[1])), x2, b2(ps[2])), x);
        }
        *c = f2(hw_cos(x.x), hw_cos(x.y));
    } else {
        sincos2<PHC>(x, s, c);
    }
}

// Packed mixed precision in wavenumber-scaled units (as regular_dp0_mixed2_tile).
// Per point pair, with g = w (d'.n) / r'^2 and the shared factors
// h1 = cos / r' + sin, h2 = cos - sin / r', the double-layer part of an entry
// is -g h1 + i g h2 (times kappa^2); the two entries differ only in (d'.n).
//
// Per element pair: the centroid offset D and |D|^2 in FP64 (r_c' for the
// phase), FP32 copies for the point-pair terms; elements whose centroids are
// farther apart than prm.near_r cannot share a vertex, so the vertex test
// runs only for near pairs; the pair phase exp(i r_c') by phase_reduced32.
// The six test points form two orbits of equal weight (w_a for points 0-2,
// w_b for 3-5, the order-4 rule): the FP32 sums of the first orbit are scaled
// by w_a / w_b when the second begins, and everything is converted to FP64
// once, times w_b.
// CK: a complex wavenumber k = kr + i ki in units of 1/kr: the amplitude e^{-beta r'} (beta = ki / kr)
// split like the phase, e^{-beta theta} per point pair by __expf and e^{-beta r_c'} per element pair by
// exp_neg_reduced; the double-layer factor (i k r - 1) = -(1 + beta r') + i r' turns 1 / r' into
// 1 / r' + beta in h1 and h2.
template <int K, int PHC, bool STRIPE = false, bool CK = false>
__device__ __forceinline__ void regular_dp0_mixed_sym_tile(const RegParams &prm, const QuadRule &rule,
                                                         int64_t tile_x, int64_t t0, int rows, TestBlock32q &sb) {
    using ST = SymTraits<K>;
    static_assert(!CK || ST::helm, "complex wavenumber: the Helmholtz kernels");
    constexpr int NP = NQ6 / 2;
    // units of 1/kappa: Re k (Helmholtz), omega (modified Helmholtz), 1 (Laplace); callers guarantee kappa > 0
    const double kap = ST::helm || ST::modhelm ? prm.p[0] : 1.0;
    const double betd = CK ? prm.p[1] / prm.p[0] : 0.0;
    const float2 bet2 = b2((float)betd);
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
            const float m2 = fmaf(o2, o2, fmaf(o1, o1, o0 * o0));
            sb.mxy[idx][p] = make_float4(-2.f * o0, -2.f * o0, -2.f * o1, -2.f * o1);
            sb.mzw[idx][p] = make_float4(-2.f * o2, -2.f * o2, m2, m2);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.c[idx][d] = c[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        sb.n[idx] = make_float4((float)g.n[0], (float)g.n[1], (float)g.n[2], 0.f);
        sb.ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = tile_x * DP0_THREADS + threadIdx.x;
    if (si < prm.ntrial && t0 <= si) {
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    float2 yx[NP], yyy[NP], yz[NP], yy2[NP], wq2[NP];
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
        wq2[j] = f2(rule.wf[2 * j], rule.wf[2 * j + 1]);
    }
    const double ek_r = (K == BEMPPCUDA_HELMHOLTZ_COMBINED) ? kap * prm.p[2] : kap;
    const double ek_i = (K == BEMPPCUDA_HELMHOLTZ_COMBINED) ? kap * prm.p[3] : 0.0;
    const double k2d = kap * kap;
    // test-point weights: w_b for the second orbit, w_a / w_b applied in FP32 to the first
    const double wb = rule.w[NQ6 - 1];
    const float2 rho2 = b2((float)(rule.w[0] / wb));
    // centroid distances below near_r (scaled) may belong to vertex-sharing pairs
    const double near2 = prm.near_r > 0.0 ? (kap * prm.near_r) * (kap * prm.near_r) : 1e300;

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        if (row > si) break;
        const double D0 = kap * (sc[0] - sb.c[tt][0]), D1 = kap * (sc[1] - sb.c[tt][1]),
                     D2 = kap * (sc[2] - sb.c[tt][2]);
        const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
        const bool adj = row == si ||
                         (prm.grids_identical && rc2 <= near2 && shares_vertex(sb.v[tt], sv0, sv1, sv2));
        double a_re = 0.0, a_im = 0.0, b_re = 0.0, b_im = 0.0;  // A_ij, A_ji
        if (!adj) {
            const double rc = rc2 * rsqrt64(rc2);
            float ph_s = 0.f, ph_c = 1.f;
            if (ST::helm) phase_reduced32(rc, &ph_s, &ph_c);
            // e^{-beta r_c'} (complex k), e^{-r_c'} (modified Helmholtz)
            const double amp = CK ? exp_neg_reduced(betd * rc) : (ST::modhelm ? exp_neg_reduced(rc) : 1.0);
            const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
            const float2 rcf2 = b2((float)rc), rc2f2 = b2((float)rc2);
            // k (y - x).n_j = cp_p (y lies in the plane of j, so (y - c_j).n_j = 0) and
            // k (x - y).n_i = ynt_q ((x - c_i).n_i = 0): one factor per test point, one per trial point
            float nh0 = 0.f, nh1 = 0.f, nh2 = 0.f, Dn = 0.f;
            float2 ynt[NP];
            if (ST::dlp_part) {
                const float4 tn = sb.n[tt];
                const float2 Dt = b2(-fmaf(D2f, tn.z, fmaf(D1f, tn.y, D0f * tn.x)));
#pragma unroll
                for (int j = 0; j < NP; ++j)
                    ynt[j] = fma2(yz[j], b2(-tn.z), fma2(yyy[j], b2(-tn.y), fma2(yx[j], b2(-tn.x), Dt)));
                Dn = fmaf(D2f, sn2, fmaf(D1f, sn1, D0f * sn0));
                nh0 = 0.5f * sn0;
                nh1 = 0.5f * sn1;
                nh2 = 0.5f * sn2;
            }
            const float2 D0d = b2(2.f * D0f), D1d = b2(2.f * D1f), D2d = b2(2.f * D2f);
            float2 A[NP];
#pragma unroll
            for (int j = 0; j < NP; ++j) A[j] = fma2(D2d, yz[j], fma2(D1d, yyy[j], fma2(D0d, yx[j], yy2[j])));
            float2 s0r = b2(0.f), s0i = b2(0.f), ur = b2(0.f), ui = b2(0.f), vr = b2(0.f), vi = b2(0.f);
#pragma unroll
            for (int p = 0; p < NQ6; ++p) {
                if (p == NQ6 / 2) {  // second orbit: the first orbit's sums times w_a / w_b
                    s0r = mul2(s0r, rho2);
                    s0i = mul2(s0i, rho2);
                    ur = mul2(ur, rho2);
                    ui = mul2(ui, rho2);
                    vr = mul2(vr, rho2);
                    vi = mul2(vi, rho2);
                }
                const float4 mxy = sb.mxy[tt][p], mzw = sb.mzw[tt][p];
                const float2 mx = f2(mxy.x, mxy.y), my = f2(mxy.z, mxy.w), mz = f2(mzw.x, mzw.y);
                const float2 Bp2 = b2(fmaf(D2f, mzw.x, fmaf(D1f, mxy.z, fmaf(D0f, mxy.x, mzw.z))));
                float2 cp2 = b2(0.f);
                if (ST::dlp_part) cp2 = b2(fmaf(mzw.x, nh2, fmaf(mxy.z, nh1, fmaf(mxy.x, nh0, Dn))));
                float2 pur = b2(0.f), pui = b2(0.f);  // sum over q of the A_ij double-layer factor, times cp per p
#pragma unroll
                for (int j = 0; j < NP; ++j) {
                    const float2 sdot = fma2(yz[j], mz, fma2(yyy[j], my, fma2(yx[j], mx, add2(A[j], Bp2))));
                    const float2 r2 = add2(rc2f2, sdot);
                    const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                    const float2 f = mul2(wq2[j], rinv);
                    if (!ST::helm) {
                        // modified Helmholtz: e^{-theta} per pair (e^{-r_c'} per element pair), the double
                        // layers' (1 + r') e^{-theta}
                        float2 am = b2(1.f), am1 = b2(1.f);
                        if (ST::modhelm) {
                            const float2 den = fma2(r2, rinv, rcf2);
                            const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                            am = f2(__expf(-th.x), __expf(-th.y));
                            am1 = mul2(am, fma2(r2, rinv, b2(1.f)));
                        }
                        if (ST::slp_part) s0r = ST::modhelm ? fma2(f, am, s0r) : add2(f, s0r);
                        if (ST::dlp_part) {
                            float2 fr = mul2(mul2(f, rinv), rinv);
                            if (ST::modhelm) fr = mul2(fr, am1);
                            pur = add2(fr, pur);
                            vr = fma2(fr, ynt[j], vr);
                        }
                    } else {
                        const float2 den = fma2(r2, rinv, rcf2);
                        const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                        float2 sn, cs;
                        sincos2_sym<PHC>(th, &sn, &cs);
                        if (CK) {
                            const float2 am = f2(__expf(-bet2.x * th.x), __expf(-bet2.x * th.y));
                            cs = mul2(cs, am);
                            sn = mul2(sn, am);
                        }
                        if (ST::slp_part) {
                            s0r = fma2(f, cs, s0r);
                            s0i = fma2(f, sn, s0i);
                        }
                        if (ST::dlp_part) {
                            const float2 fr = mul2(f, rinv);
                            const float2 rb = CK ? add2(rinv, bet2) : rinv;  // 1 / r' (+ beta)
                            const float2 h1 = fma2(rb, cs, sn);
                            const float2 h2 = fma2(f2(-rb.x, -rb.y), sn, cs);
                            const float2 gt = mul2(fr, ynt[j]);
                            pur = fma2(fr, h1, pur);
                            pui = fma2(fr, h2, pui);
                            vr = fma2(gt, h1, vr);
                            vi = fma2(gt, h2, vi);
                        }
                    }
                }
                if (ST::dlp_part) {
                    ur = fma2(cp2, pur, ur);
                    if (ST::helm) ui = fma2(cp2, pui, ui);
                }
            }
            // entry = w_b [kappa eta S0 + kappa^2 (-h1 sum + i h2 sum)], rotated by exp(i r_c') and scaled
            double sr = 0.0, sim = 0.0;
            if (ST::slp_part) {
                const double xr = (double)(s0r.x + s0r.y), xi = (double)(s0i.x + s0i.y);
                sr = fma(ek_r, xr, -ek_i * xi);
                sim = fma(ek_r, xi, ek_i * xr);
            }
            double dr = 0.0, di = 0.0, er = 0.0, ei = 0.0;
            if (ST::dlp_part) {
                dr = -k2d * (double)(ur.x + ur.y);
                er = -k2d * (double)(vr.x + vr.y);
                if (ST::helm) {
                    di = k2d * (double)(ui.x + ui.y);
                    ei = k2d * (double)(vi.x + vi.y);
                }
            }
            if (ST::swap) {
                a_re = er;
                a_im = ei;
                b_re = dr;
                b_im = di;
            } else {
                a_re = sr + dr;
                a_im = sim + di;
                b_re = sr + er;
                b_im = sim + ei;
            }
            const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie * wb * amp;
            const double pc = (double)ph_c, ps = (double)ph_s;
            double tr = a_re * pc - a_im * ps;
            a_im = (a_re * ps + a_im * pc) * scale;
            a_re = tr * scale;
            tr = b_re * pc - b_im * ps;
            b_im = (b_re * ps + b_im * pc) * scale;
            b_re = tr * scale;
        }
        store_pair<STRIPE>(prm, row, si, adj, a_re, a_im, b_re, b_im);
    }
    }
    __syncthreads();
}

}  // namespace bc
