// Regular pairs of scalar operators on linear (P1 / DP1) and mixed P0 / P1
// spaces, 6-point rule: the kernels of numba_kernels.py:980-1074
// (default_scalar_regular_kernel) and the hypersingular ones of :1078-1467.
//
// One thread per trial element, 32 test elements staged in shared memory (as
// the DP0 tiles).  Per test point p the trial sums
//   T_j(p) = sum_q w_q K(x_p, y_q) psi_j(q)          (j < NS)
// are formed first, then L_ij += w_p phi_i(p) T_j(p), so a point pair costs NS
// complex FMAs instead of NT x NS.  Hypersingular operators reuse the single-
// layer sums: with constant surface curls per element,
//   L_ij = (curl_i . curl_j) S - c (n_t . n_s) M_ij,  S = sum_j T_j summed over p
// (the P1 shape functions add up to 1), c = k^2 (Helmholtz), 0 (Laplace).
// exp(ikr) is factored about the centroid distance as in the DP0 kernels
// (phase classes 1, 2); class 3 is a complex wavenumber k = kr + i ki:
// exp(i kr r) from the reduced sine / cosine times exp(-ki r), the double-layer
// factor (ikr - 1) / r = (-1/r - ki) + i kr, and -k^2 complex in the
// hypersingular operator.  The symmetric and skew sweeps hold for complex k
// (G(x, y) = G(y, x)).  Modified Helmholtz, G = exp(-w r) / (4 pi r) with
// w = p[0] > 0, is real: the Laplace kernels times exp(-w r) (single layer) or
// exp(-w r) (1 + w r) (double layers), and +w^2 (n_t . n_s) in the
// hypersingular operator.
// The NT x NS block is added to the matrix with FP64 atomics (l2g, multipliers).
// SYM (the same space on both sides): only pairs i < j (support positions) are
// evaluated and each gives the blocks at (i, j) and (j, i).  Single layer and
// hypersingular: the kernel is symmetric in x and y and so is the curl
// product, so the second block is the transpose of the first; into a zeroed
// result (defer_transpose) only the first is added and the host forms
// A = U + U^T afterwards (the regular diagonal is zero: a pair that reaches
// entry (I, I) shares vertex I and is singular).  Double and
// adjoint double layer: with d = y - x, the double layer of the transposed
// pair (test j, trial i) is the adjoint double layer of (i, j) --
//   (ikr - 1) e^{ikr} ((x - y) . n_i) / r^3 = -(ikr - 1) e^{ikr} (d . n_i) / r^3
// -- so both blocks share r, the phase and (ikr - 1) e^{ikr} / r^2 and differ
// in the normal of the dot product (the trial normal for the double layer).
#pragma once

#include "dp0.cuh"

namespace bc {

constexpr int P1_TCHUNK = 32;

struct TestBlockP1 {
    double x[P1_TCHUNK][NQ6][3];
    double n[P1_TCHUNK][3];
    double c[P1_TCHUNK][3];
    double curl[P1_TCHUNK][3][3];
    double ie[P1_TCHUNK];
    double mult[P1_TCHUNK][3];  // local multipliers of the test functions
    int64_t row[P1_TCHUNK][3];  // their global dofs
    int v[P1_TCHUNK][3];
};

// CTAs per SM the P1 kernel is compiled for: no cap (184-214 registers) beat
// a cap of 3 on the double layer and hypersingular operators at L5.
#ifndef BC_P1_MIN_BLOCKS
#define BC_P1_MIN_BLOCKS 1
#endif

template <int ASM, int K, int NT, int NS, int PHC, bool SYM>
__global__ void __launch_bounds__(DP0_THREADS, BC_P1_MIN_BLOCKS) regular_p1(RegParams prm, QuadRule rule) {
    constexpr bool HYP = (ASM == BEMPPCUDA_ASM_LAPLACE_HYP || ASM == BEMPPCUDA_ASM_HELM_HYP ||
                          ASM == BEMPPCUDA_ASM_MODHELM_HYP);
    constexpr bool HELM = (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                           K == BEMPPCUDA_HELMHOLTZ_ADLP);
    constexpr bool MH = (K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_MODHELM_ADLP);
    constexpr bool DL = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_MODHELM_DLP);
    constexpr bool AD = (K == BEMPPCUDA_LAPLACE_ADLP || K == BEMPPCUDA_HELMHOLTZ_ADLP || K == BEMPPCUDA_MODHELM_ADLP);
    constexpr bool PH = HELM && (PHC == 1 || PHC == 2);
    constexpr bool CK = HELM && PHC == 3;
    static_assert(!SYM || NT == NS, "the symmetric sweep needs one space on both sides");
    constexpr bool SKEW = SYM && (DL || AD);  // the transposed block uses the other element's normal
    __shared__ TestBlockP1 sb;

    const int64_t t0 = (int64_t)blockIdx.y * P1_TCHUNK;
    if (SYM && t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;  // below the diagonal
    const int tcount = (int)min((int64_t)P1_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        for (int p = 0; p < NQ6; ++p) to_global(g, rule.x[p], rule.y[p], sb.x[idx][p]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.n[idx][d] = g.n[d];
            sb.c[idx][d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            sb.mult[idx][i] = prm.tmult[t * NT + i];
            sb.row[idx][i] = prm.tl2g[t * NT + i];
        }
        if (HYP) {
            double cu[3][3];
            surface_curls(prm.tg, prm.tne, t, g.n, cu);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int d = 0; d < 3; ++d) sb.curl[idx][i][d] = cu[i][d];
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
    double y[NQ6][3];
#pragma unroll
    for (int q = 0; q < NQ6; ++q) to_global(gs, rule.x[q], rule.y[q], y[q]);
    double sc[3] = {0.0, 0.0, 0.0};
    if (PH)
#pragma unroll
        for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    double curl_s[3][3];
    if (HYP) surface_curls(prm.sg, prm.sne, s, gs.n, curl_s);
    // trial / test shape values times the weights (constant operands from the rule)
    const auto psw = [&](int q, int j) -> double { return NS == 1 ? rule.w[q] : rule.sw[q][j]; };
    const double kr = prm.p[0], ki = CK ? prm.p[1] : 0.0;
    // the trial dofs and multipliers stay in registers for the whole tile
    int64_t scol[NS];
    double smul[NS];
#pragma unroll
    for (int j = 0; j < NS; ++j) {
        scol[j] = prm.sl2g[s * NS + j];
        smul[j] = prm.smult[s * NS + j];
    }
    // (y_q - v0_s).n_s, the split of the double-layer normal term about the trial vertex 0
    double ynv[NQ6];
    if (DL && !SKEW)
#pragma unroll
        for (int q = 0; q < NQ6; ++q)
            ynv[q] = fma(y[q][2] - gs.v0[2], gs.n[2], fma(y[q][1] - gs.v0[1], gs.n[1], (y[q][0] - gs.v0[0]) * gs.n[0]));

    for (int tt = 0; tt < tcount; ++tt) {
        if (SYM && t0 + tt >= si) break;  // rows increase with tt
        if (prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2)) continue;
        const int64_t t = prm.tsup[t0 + tt];
        // SKEW: the normal factors by the plane property (a quadrature point lies in its own element's
        // plane): (y_q - x_p).n_s = (v0_s - x_p).n_s, one value per test point (xn below), and
        // (x_p - y_q).n_t = (c_t - y_q).n_t, one value per trial point
        double mdt[SKEW ? NQ6 : 1];
        if (SKEW)
#pragma unroll
            for (int q = 0; q < NQ6; ++q)
                mdt[q % (SKEW ? NQ6 : 1)] =
                    fma(sb.c[tt][2] - y[q][2], sb.n[tt][2],
                        fma(sb.c[tt][1] - y[q][1], sb.n[tt][1], (sb.c[tt][0] - y[q][0]) * sb.n[tt][0]));
        double rc = 0.0, krc = 0.0, ph_s = 0.0, ph_c = 1.0;
        if (PH) {
            const double D0 = sc[0] - sb.c[tt][0], D1 = sc[1] - sb.c[tt][1], D2 = sc[2] - sb.c[tt][2];
            rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
            krc = kr * rc;
            sincos_cw64(krc, &ph_s, &ph_c);
        }
        double lre[NT][NS], lim[NT][NS];
        double ure[SKEW ? NT : 1][SKEW ? NS : 1], uim[SKEW ? NT : 1][SKEW ? NS : 1];  // SKEW: block of (j, i)
#pragma unroll
        for (int i = 0; i < NT; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) lre[i][j] = lim[i][j] = 0.0;
        if (SKEW)
#pragma unroll
            for (int i = 0; i < NT; ++i)
#pragma unroll
                for (int j = 0; j < NS; ++j) ure[i % (SKEW ? NT : 1)][j % (SKEW ? NS : 1)] = uim[i % (SKEW ? NT : 1)][j % (SKEW ? NS : 1)] = 0.0;
        double sre = 0.0, sim = 0.0;  // HYP: sum_pq w G
        for (int p = 0; p < NQ6; ++p) {
            const double x0 = sb.x[tt][p][0], x1 = sb.x[tt][p][1], x2 = sb.x[tt][p][2];
            double xn = 0.0;
            if (DL || SKEW) xn = fma(gs.v0[2] - x2, gs.n[2], fma(gs.v0[1] - x1, gs.n[1], (gs.v0[0] - x0) * gs.n[0]));
            double tre[NS], tim[NS], vre[SKEW ? NS : 1], vim[SKEW ? NS : 1];
#pragma unroll
            for (int j = 0; j < NS; ++j) tre[j] = tim[j] = 0.0;
            if (SKEW)
#pragma unroll
                for (int j = 0; j < NS; ++j) vre[j % (SKEW ? NS : 1)] = vim[j % (SKEW ? NS : 1)] = 0.0;
#pragma unroll
            for (int q = 0; q < NQ6; ++q) {
                const double d0 = y[q][0] - x0, d1 = y[q][1] - x1, d2 = y[q][2] - x2;
                const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                const double rinv = rsqrt64(r2);
                double kre, kim = 0.0;  // kernel value without 1/(4 pi)
                double k2re = 0.0, k2im = 0.0;  // SKEW: the transposed pair's kernel
                if (SKEW) {
                    double hre, him;  // double layer of trial normal n: (dot with n) (hre + i him)
                    if (!HELM) {
                        hre = -rinv * rinv * rinv;
                        if (MH) {
                            const double r = r2 * rinv;
                            hre *= exp(-kr * r) * fma(kr, r, 1.0);
                        }
                        him = 0.0;
                    } else {
                        const double r = r2 * rinv;
                        double sn, cs;
                        if (PH && PHC == 2)
                            sincos_half64(fma(kr, r, -krc), &sn, &cs);
                        else if (PH)
                            sincos_small64(fma(kr, r, -krc), &sn, &cs);
                        else
                            sincos_cw64(kr * r, &sn, &cs);
                        if (CK) {
                            const double am = exp(-ki * r);
                            sn *= am;
                            cs *= am;
                        }
                        const double rinv2 = rinv * rinv, rk = CK ? rinv + ki : rinv;
                        hre = -rinv2 * fma(rk, cs, kr * sn);
                        him = rinv2 * fma(kr, cs, -rk * sn);
                    }
                    // h alone (its trial-normal factor xn is applied per test point), and h times the
                    // test-normal factor of this trial point
                    kre = hre;
                    kim = him;
                    k2re = mdt[q % (SKEW ? NQ6 : 1)] * hre;
                    k2im = mdt[q % (SKEW ? NQ6 : 1)] * him;
                } else if (!HELM) {
                    if (K == BEMPPCUDA_LAPLACE_SLP) {
                        kre = rinv;
                    } else if (K == BEMPPCUDA_MODHELM_SLP) {
                        kre = exp(-kr * (r2 * rinv)) * rinv;
                    } else {
                        const double dot = DL ? ynv[q] + xn
                                              : fma(d2, sb.n[tt][2], fma(d1, sb.n[tt][1], d0 * sb.n[tt][0]));
                        kre = (DL ? -dot : dot) * rinv * rinv * rinv;
                        if (MH) {
                            const double r = r2 * rinv;
                            kre *= exp(-kr * r) * fma(kr, r, 1.0);
                        }
                    }
                } else {
                    const double r = r2 * rinv;
                    double sn, cs;
                    if (PH && PHC == 2)
                        sincos_half64(fma(kr, r, -krc), &sn, &cs);
                    else if (PH)
                        sincos_small64(fma(kr, r, -krc), &sn, &cs);
                    else
                        sincos_cw64(kr * r, &sn, &cs);
                    if (CK) {
                        const double am = exp(-ki * r);
                        sn *= am;
                        cs *= am;
                    }
                    if (K == BEMPPCUDA_HELMHOLTZ_SLP) {
                        kre = cs * rinv;
                        kim = sn * rinv;
                    } else {
                        // (ikr - 1) e^{ikr} dot / r^3 = g (-h1 + i h2), g = dot / r^2
                        const double dot = DL ? ynv[q] + xn
                                              : -fma(d2, sb.n[tt][2], fma(d1, sb.n[tt][1], d0 * sb.n[tt][0]));
                        const double g = dot * rinv * rinv, rk = rinv + ki;
                        kre = -g * fma(rk, cs, kr * sn);
                        kim = g * fma(kr, cs, -rk * sn);
                    }
                }
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    tre[j] = fma(kre, psw(q, j), tre[j]);
                    tim[j] = fma(kim, psw(q, j), tim[j]);
                }
                if (SKEW)
#pragma unroll
                    for (int j = 0; j < NS; ++j) {
                        vre[j % (SKEW ? NS : 1)] = fma(k2re, psw(q, j), vre[j % (SKEW ? NS : 1)]);
                        vim[j % (SKEW ? NS : 1)] = fma(k2im, psw(q, j), vim[j % (SKEW ? NS : 1)]);
                    }
            }
            const double wp = rule.w[p];
            const auto phw = [&](int i) -> double { return NT == 1 ? wp : rule.sw[p][i]; };
#pragma unroll
            for (int i = 0; i < NT; ++i) {
                // SKEW: the sums of h take the trial-normal factor xn of this test point; they form the
                // (i, j) block of the double layer and the transposed block of the adjoint double layer
                const double px = SKEW ? phw(i) * xn : phw(i);
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    if (!SKEW) {
                        lre[i][j] = fma(phw(i), tre[j], lre[i][j]);
                        lim[i][j] = fma(phw(i), tim[j], lim[i][j]);
                    } else {
                        constexpr int a = SKEW ? NT : 1, b = SKEW ? NS : 1;
                        // (weight, sum) of the (i, j) block and of the transposed pair's block
                        const double w1 = DL ? px : phw(i), w2 = DL ? phw(i) : px;
                        const double s1r = DL ? tre[j] : vre[j % b], s1i = DL ? tim[j] : vim[j % b];
                        const double s2r = DL ? vre[j % b] : tre[j], s2i = DL ? vim[j % b] : tim[j];
                        lre[i][j] = fma(w1, s1r, lre[i][j]);
                        lim[i][j] = fma(w1, s1i, lim[i][j]);
                        ure[i % a][j % b] = fma(w2, s2r, ure[i % a][j % b]);
                        uim[i % a][j % b] = fma(w2, s2i, uim[i % a][j % b]);
                    }
                }
            }
            if (HYP)
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    sre = fma(wp, tre[j], sre);
                    sim = fma(wp, tim[j], sim);
                }
        }
        const double scale = BC_INV_4PI * sb.ie[tt] * gs.ie;
        // hypersingular: -k^2 (n_t . n_s), complex for a complex wavenumber; +w^2 (n_t . n_s) modified
        double cpf = 0.0, cpi = 0.0;
        if (HYP && ASM == BEMPPCUDA_ASM_HELM_HYP) {
            const double nn = sb.n[tt][0] * gs.n[0] + sb.n[tt][1] * gs.n[1] + sb.n[tt][2] * gs.n[2];
            cpf = -(kr * kr - ki * ki) * nn;
            cpi = -2.0 * kr * ki * nn;
        } else if (HYP && ASM == BEMPPCUDA_ASM_MODHELM_HYP) {
            cpf = kr * kr * (sb.n[tt][0] * gs.n[0] + sb.n[tt][1] * gs.n[1] + sb.n[tt][2] * gs.n[2]);
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const double mt = sb.mult[tt][i];
            if (mt == 0.0) continue;
            const int64_t row = sb.row[tt][i];
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const double ms = smul[j];
                if (ms == 0.0) continue;
                double vr = lre[i][j], vi = lim[i][j];
                if (HYP) {
                    const double cij = sb.curl[tt][i][0] * curl_s[j][0] + sb.curl[tt][i][1] * curl_s[j][1] +
                                       sb.curl[tt][i][2] * curl_s[j][2];
                    const double lr = vr, li = vi;
                    vr = fma(cij, sre, fma(cpf, lr, -cpi * li));
                    vi = fma(cij, sim, fma(cpf, li, cpi * lr));
                }
                // SKEW: the transposed pair's own block, else the same block
                double wr = SKEW ? ure[i % (SKEW ? NT : 1)][j % (SKEW ? NS : 1)] : vr;
                double wi = SKEW ? uim[i % (SKEW ? NT : 1)][j % (SKEW ? NS : 1)] : vi;
                if (PH) {
                    const double tr = vr * ph_c - vi * ph_s;
                    vi = fma(vr, ph_s, vi * ph_c);
                    vr = tr;
                    if (SKEW) {
                        const double ur = wr * ph_c - wi * ph_s;
                        wi = fma(wr, ph_s, wi * ph_c);
                        wr = ur;
                    } else {
                        wr = vr;
                        wi = vi;
                    }
                }
                const double m = mt * ms * scale;
                const int64_t col = scol[j];
                if (prm.is_complex) {
                    double *o = reinterpret_cast<double *>(prm.result) + 2 * (row * prm.ld + col);
                    atomicAdd(o, vr * m);
                    atomicAdd(o + 1, vi * m);
                    if (SYM && (SKEW || !prm.defer_transpose)) {
                        double *ot = reinterpret_cast<double *>(prm.result) + 2 * (col * prm.ld + row);
                        atomicAdd(ot, wr * m);
                        atomicAdd(ot + 1, wi * m);
                    }
                } else {
                    atomicAdd(reinterpret_cast<double *>(prm.result) + row * prm.ld + col, vr * m);
                    if (SYM && (SKEW || !prm.defer_transpose))
                        atomicAdd(reinterpret_cast<double *>(prm.result) + col * prm.ld + row, wr * m);
                }
            }
        }
    }
}

}  // namespace bc
