// Regular pairs of the Maxwell electric and magnetic field operators on RWG /
// SNC spaces, 6-point rule: the kernels of
// numba_kernels.py:1853-1969 (maxwell_efield_regular_assembler) and
// :2151-2280 (maxwell_mfield_regular_assembler).
//
// Basis: b_i = J r_i / |J| with the reference RWG functions
// r_i = (xi - a_i, eta - b_i), (a, b) = (0, 1), (1, 0), (0, 0)
// (shapesets.py:95-102; SNC evaluates the same values), so the integration
// elements of the quadrature cancel and, with G = exp(ikr) / (4 pi r),
//   EFIE_ij = sum_pq w_p w_q G [-ik (J_t r_i(p)) . (J_s r_j(q)) - 4 / (ik)]
//   MFIE_ij = sum_pq w_p w_q G (ikr - 1) / r^2 (x - y) . (J_t r_i(p) x J_s r_j(q)),
// each times the two edge lengths and multipliers.  Write J_t r_i(p) =
// w_t(p) - c_ti with w_t(p) = x_p - v0_t = J_t (xi_p, eta_p) and
// c_ti = J_t (a_i, b_i) (c_t2 = 0); likewise on the trial side.  Then no
// per-function work is left inside the point loops:
//  EFIE: with the nine moments M[u][v] = sum_pq w_p w_q G u(p) v(q),
//        u, v in {1, xi, eta} (accumulated as the P1 kernel accumulates its sums),
//          sum_pq w w G (J_t r_i) . (J_s r_j) = P - c_sj . V_t - c_ti . V_s + (c_ti . c_sj) M[1][1],
//        P = sum_ab (J_ta . J_sb) M[e_a][e_b], V_t = sum_a J_ta M[e_a][1],
//        V_s = sum_b J_sb M[1][e_b]  (e_0 = xi, e_1 = eta).
//  MFIE: with P_ti = v0_t + c_ti the vertex function i points away from, J_t r_i(p) = x_p - P_ti,
//        so (x - y) . (J_t r_i x J_s r_j) = (P_ti - P_sj) . (J_t r_i x J_s r_j): the same nine
//        moments, of H = G (ikr - 1) / r^2 in place of G, give the block (mfie_block_moments:
//        MFIE_ij = sum_ab det(P_ti - P_sj, J_t^a, J_s^b) times the moments shifted by (a_i, b_i),
//        (a_j, b_j)).  The singular kernel sums, with H = w_p w_q G (ikr - 1) / r^2, d = x - y,
//          B(p) = sum_q H (w_s(q) x d),  C(p) = sum_q H d,
//          MFIE_ij = PB - c_sj . PC - c_ti . QB + c_ti . (c_sj x QC),
//        PB = sum_p w_t(p) . B(p), PC = sum_p C(p) x w_t(p), QB = sum_p B(p), QC = sum_p C(p).
// exp(ikr) is factored about the centroid distance as in the DP0 / P1 kernels
// (phase classes 1, 2).  Class 3 is a complex wavenumber k = kr + i ki:
// exp(ikr) = exp(i kr r) exp(-ki r) per point pair, (ikr - 1) = -(1 + ki r) + i kr r,
// and -ik, -4 / (ik) = 4i conj(k) / |k|^2 as complex factors per element pair.
// SYM (test and trial spaces with the same dof maps on one grid, as RWG and
// SNC are): both operators are symmetric under exchanging the pair's
// elements (G is symmetric; for MFIE both d and the cross product change
// sign), so pairs i < j are evaluated once and added at (i, j) and (j, i).
#pragma once

#include "dp0.cuh"

namespace bc {

constexpr int RWG_TCHUNK = 32;

struct TestBlockRWG {
    double x[RWG_TCHUNK][NQ6][3];
    double j0[RWG_TCHUNK][3];
    double j1[RWG_TCHUNK][3];
    double c[RWG_TCHUNK][3];
    double v0[RWG_TCHUNK][3];   // vertex 0 (MFIE moments)
    double fac[RWG_TCHUNK][3];  // edge length times multiplier of each test function
    int64_t row[RWG_TCHUNK][3];
    int v[RWG_TCHUNK][3];
};

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
    return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0]));
}

// EFIE block of an element pair from its nine moments M[u][v] = sum_pq w_p w_q G u(p) v(q), u, v in
// {1, xi, eta} (index 0, 1, 2; G times 4 pi, any phase factor of the pair left out): the formula of the
// header comment, for real k (CK false) or complex k = kr + i ki.
template <bool CK>
__device__ __forceinline__ void efie_block(const double mre[3][3], const double mim[3][3], const double tj0[3],
                                           const double tj1[3], const double sj0[3], const double sj1[3], double kr,
                                           double ki, double blk_re[3][3], double blk_im[3][3]) {
    // c_t = (J_t (0, 1), J_t (1, 0), 0) = (j1_t, j0_t, 0); likewise c_s
    const double *ctv[2] = {tj1, tj0};
    const double *csv[2] = {sj1, sj0};
    // P, V_t, V_s from the moments (index 0 = 1, 1 = xi, 2 = eta)
    const double D00 = dot3(tj0, sj0), D01 = dot3(tj0, sj1), D10 = dot3(tj1, sj0), D11 = dot3(tj1, sj1);
    const double pr = D00 * mre[1][1] + D01 * mre[1][2] + D10 * mre[2][1] + D11 * mre[2][2];
    const double pi = D00 * mim[1][1] + D01 * mim[1][2] + D10 * mim[2][1] + D11 * mim[2][2];
    double vtr[3], vti[3], vsr[3], vsi[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        vtr[c] = fma(tj0[c], mre[1][0], tj1[c] * mre[2][0]);
        vti[c] = fma(tj0[c], mim[1][0], tj1[c] * mim[2][0]);
        vsr[c] = fma(sj0[c], mre[0][1], sj1[c] * mre[0][2]);
        vsi[c] = fma(sj0[c], mim[0][1], sj1[c] * mim[0][2]);
    }
    // -ik E1 - 4 / (ik) M11, 1 / (ik) = -i / k
    const double m11r = mre[0][0], m11i = mim[0][0];
    // complex k: -4 / (ik) M11 = 4 (ki + i kr) / |k|^2 M11, one value per pair
    double c1r = 0.0, c1i = 0.0;
    if (CK) {
        const double g4 = 4.0 / fma(kr, kr, ki * ki);
        c1r = g4 * fma(ki, m11r, -kr * m11i);
        c1i = g4 * fma(kr, m11r, ki * m11i);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double er = pr, ei = pi;
            if (j < 2) {
                er -= dot3(csv[j], vtr);
                ei -= dot3(csv[j], vti);
            }
            if (i < 2) {
                er -= dot3(ctv[i], vsr);
                ei -= dot3(ctv[i], vsi);
            }
            if (i < 2 && j < 2) {
                const double cc = dot3(ctv[i], csv[j]);
                er = fma(cc, m11r, er);
                ei = fma(cc, m11i, ei);
            }
            // -ik (er + i ei) = k ei - i k er;  -(4 / (ik)) M11 = (4i / k) M11 = -4 m11i / k + i 4 m11r / k
            if (CK) {
                // -ik (er + i ei) = (kr ei + ki er) + i (ki ei - kr er)
                blk_re[i][j] = fma(kr, ei, fma(ki, er, c1r));
                blk_im[i][j] = fma(ki, ei, fma(-kr, er, c1i));
            } else {
                blk_re[i][j] = fma(kr, ei, -4.0 * m11i / kr);
                blk_im[i][j] = fma(-kr, er, 4.0 * m11r / kr);
            }
        }
}

// MFIE block of an element pair from its four sums (any phase factor of the pair left out):
// MFIE_ij = PB - c_sj . PC - c_ti . QB + c_ti . (c_sj x QC), the formula of the header comment.
__device__ __forceinline__ void mfie_block(double pbr, double pbi, const double pcr[3], const double pci[3],
                                           const double qbr[3], const double qbi[3], const double qcr[3],
                                           const double qci[3], const double tj0[3], const double tj1[3],
                                           const double sj0[3], const double sj1[3], double blk_re[3][3],
                                           double blk_im[3][3]) {
    const double *ctv[2] = {tj1, tj0};
    const double *csv[2] = {sj1, sj0};
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double vr = pbr, vi = pbi;
            if (j < 2) {
                vr -= dot3(csv[j], pcr);
                vi -= dot3(csv[j], pci);
            }
            if (i < 2) {
                vr -= dot3(ctv[i], qbr);
                vi -= dot3(ctv[i], qbi);
                if (j < 2) {
                    // c_ti . (c_sj x QC) = QC . (c_ti x c_sj)
                    double cx[3];
                    cx[0] = ctv[i][1] * csv[j][2] - ctv[i][2] * csv[j][1];
                    cx[1] = ctv[i][2] * csv[j][0] - ctv[i][0] * csv[j][2];
                    cx[2] = ctv[i][0] * csv[j][1] - ctv[i][1] * csv[j][0];
                    vr += dot3(cx, qcr);
                    vi += dot3(cx, qci);
                }
            }
            blk_re[i][j] = vr;
            blk_im[i][j] = vi;
        }
}

// MFIE block of an element pair from the nine moments M[u][v] = sum_pq w_p w_q H u(p) v(q), u, v in
// {1, xi, eta} (index 0, 1, 2; H = e^{ikr} (ikr - 1) / r^3 times 4 pi, any phase factor of the pair left
// out) and the two elements' vertex 0 and Jacobian columns: the formula of the header comment.
__device__ __forceinline__ void mfie_block_moments(const double mre[3][3], const double mim[3][3],
                                                   const double tv0[3], const double tj0[3], const double tj1[3],
                                                   const double sv0[3], const double sj0[3], const double sj1[3],
                                                   double blk_re[3][3], double blk_im[3][3]) {
    const double *tJ[2] = {tj0, tj1}, *sJ[2] = {sj0, sj1};
    // C_ab = J_t^a x J_s^b, and the vertex offsets P - v0 = J (a_i, b_i): (j1, j0, 0) per function
    double C[2][2][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            C[a][b][0] = tJ[a][1] * sJ[b][2] - tJ[a][2] * sJ[b][1];
            C[a][b][1] = tJ[a][2] * sJ[b][0] - tJ[a][0] * sJ[b][2];
            C[a][b][2] = tJ[a][0] * sJ[b][1] - tJ[a][1] * sJ[b][0];
        }
    constexpr int oa[3] = {0, 1, 0}, ob[3] = {1, 0, 0};  // (a_i, b_i)
    // det(P_ti - P_sj, C_ab) = (v0_t - v0_s + J_t o_i - J_s o_j) . C_ab
    double e[2][2], ti[3][2][2], sj[3][2][2];
    const double dv[3] = {tv0[0] - sv0[0], tv0[1] - sv0[1], tv0[2] - sv0[2]};
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            e[a][b] = dot3(dv, C[a][b]);
            const double t0 = dot3(tj1, C[a][b]), t1 = dot3(tj0, C[a][b]);
            const double s0 = dot3(sj1, C[a][b]), s1 = dot3(sj0, C[a][b]);
            ti[0][a][b] = t0;
            ti[1][a][b] = t1;
            ti[2][a][b] = 0.0;
            sj[0][a][b] = s0;
            sj[1][a][b] = s1;
            sj[2][a][b] = 0.0;
        }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        // test side shifted moments: Mt[a][v] = M[1 + a][v] - o_ia M[0][v]
        double mtr[2][3], mti[2][3];
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            const int o = a == 0 ? oa[i] : ob[i];
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                mtr[a][v] = o ? mre[1 + a][v] - mre[0][v] : mre[1 + a][v];
                mti[a][v] = o ? mim[1 + a][v] - mim[0][v] : mim[1 + a][v];
            }
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double vr = 0.0, vi = 0.0;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const int o = b == 0 ? oa[j] : ob[j];
                    const double nr = o ? mtr[a][1 + b] - mtr[a][0] : mtr[a][1 + b];
                    const double ni = o ? mti[a][1 + b] - mti[a][0] : mti[a][1 + b];
                    const double det = e[a][b] + ti[i][a][b] - sj[j][a][b];
                    vr = fma(det, nr, vr);
                    vi = fma(det, ni, vi);
                }
            blk_re[i][j] = vr;
            blk_im[i][j] = vi;
        }
    }
}

template <int ASM, int PHC, bool SYM>
__global__ void __launch_bounds__(DP0_THREADS) regular_rwg(RegParams prm, QuadRule rule) {
    constexpr bool EFIE = ASM == BEMPPCUDA_ASM_EFIE;
    constexpr bool PH = PHC == 1 || PHC == 2;
    constexpr bool CK = PHC == 3;
    __shared__ TestBlockRWG sb;

    // test elements per CTA: ceil(ntest / gridDim.y) <= RWG_TCHUNK (the launch picks the row blocks)
    const int rows = (int)((prm.ntest + gridDim.y - 1) / gridDim.y);
    const int64_t t0 = (int64_t)blockIdx.y * rows;
    if (SYM && t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;  // below the diagonal
    const int tcount = (int)min((int64_t)rows, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, 1.0, g);
        for (int p = 0; p < NQ6; ++p) to_global(g, rule.x[p], rule.y[p], sb.x[idx][p]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            sb.j0[idx][d] = g.j0[d];
            sb.j1[idx][d] = g.j1[d];
            sb.c[idx][d] = __ldg(prm.tg + (22 + d) * prm.tne + t);
            sb.v0[idx][d] = g.v0[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            sb.fac[idx][i] = prm.tmult[t * 3 + i] * edge_length(prm.tg, prm.tne, t, i);
            sb.row[idx][i] = prm.tl2g[t * 3 + i];
        }
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    // trial points as offsets from the trial vertex 0: w_s(q) = J_s (xi_q, eta_q)
    double ws[NQ6][3];
#pragma unroll
    for (int q = 0; q < NQ6; ++q)
#pragma unroll
        for (int d = 0; d < 3; ++d) ws[q][d] = fma(gs.j1[d], rule.y[q], gs.j0[d] * rule.x[q]);
    double sc[3] = {0.0, 0.0, 0.0};
    if (PH)
#pragma unroll
        for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    int64_t scol[3];
    double sfac[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        scol[j] = prm.sl2g[s * 3 + j];
        sfac[j] = prm.smult[s * 3 + j] * edge_length(prm.sg, prm.sne, s, j);
    }
    const double kr = prm.p[0], ki = CK ? prm.p[1] : 0.0;

    for (int tt = 0; tt < tcount; ++tt) {
        if (SYM && t0 + tt >= si) break;  // rows increase with tt
        if (prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2)) continue;
        double krc = 0.0, ph_s = 0.0, ph_c = 1.0;
        if (PH) {
            const double D0 = sc[0] - sb.c[tt][0], D1 = sc[1] - sb.c[tt][1], D2 = sc[2] - sb.c[tt][2];
            krc = kr * sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
            sincos_cw64(krc, &ph_s, &ph_c);
        }
        const double tj0[3] = {sb.j0[tt][0], sb.j0[tt][1], sb.j0[tt][2]};
        const double tj1[3] = {sb.j1[tt][0], sb.j1[tt][1], sb.j1[tt][2]};
        // moments M[u][v] = sum_pq w_p w_q K u(p) v(q), u, v in {1, xi, eta}, of K = G (EFIE) or
        // H = G (ikr - 1) / r^2 (MFIE), both times 4 pi and without the pair's phase factor
        double mre[3][3], mim[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) mre[a][b] = mim[a][b] = 0.0;
        for (int p = 0; p < NQ6; ++p) {
            // x_p relative to the trial vertex 0: d = xs - w_s(q)
            const double xs[3] = {sb.x[tt][p][0] - gs.v0[0], sb.x[tt][p][1] - gs.v0[1], sb.x[tt][p][2] - gs.v0[2]};
            double tre[3] = {0.0, 0.0, 0.0}, tim[3] = {0.0, 0.0, 0.0};  // sum_q w_q K v(q)
#pragma unroll
            for (int q = 0; q < NQ6; ++q) {
                const double d[3] = {xs[0] - ws[q][0], xs[1] - ws[q][1], xs[2] - ws[q][2]};
                const double r2 = dot3(d, d);
                const double rinv = rsqrt64(r2);
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
                // EFIE: G 4 pi = (cs + i sn) / r; MFIE: H 4 pi = (cs + i sn)(-(1 + ki r) + i k r) / r^3
                // (the phase exp(ik r_c) and 1 / (4 pi) are applied per pair)
                double gr, gi;
                if (EFIE) {
                    gr = cs * rinv;
                    gi = sn * rinv;
                } else {
                    const double f = rinv * rinv * rinv, kq = kr * r;
                    const double a = CK ? fma(ki, r, 1.0) : 1.0;
                    gr = -fma(kq, sn, a * cs) * f;
                    gi = fma(kq, cs, -a * sn) * f;
                }
                const double v[3] = {rule.w[q], rule.sw[q][1], rule.sw[q][2]};  // w_q (1, xi_q, eta_q)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    tre[b] = fma(gr, v[b], tre[b]);
                    tim[b] = fma(gi, v[b], tim[b]);
                }
            }
            const double u[3] = {rule.w[p], rule.sw[p][1], rule.sw[p][2]};  // w_p (1, xi_p, eta_p)
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    mre[a][b] = fma(u[a], tre[b], mre[a][b]);
                    mim[a][b] = fma(u[a], tim[b], mim[a][b]);
                }
        }
        double blk_re[3][3], blk_im[3][3];
        if (EFIE) {
            efie_block<CK>(mre, mim, tj0, tj1, gs.j0, gs.j1, kr, ki, blk_re, blk_im);
        } else {
            const double tv0[3] = {sb.v0[tt][0], sb.v0[tt][1], sb.v0[tt][2]};
            mfie_block_moments(mre, mim, tv0, tj0, tj1, gs.v0, gs.j0, gs.j1, blk_re, blk_im);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double ft = sb.fac[tt][i] * BC_INV_4PI;
            if (ft == 0.0) continue;
            const int64_t row = sb.row[tt][i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double m = ft * sfac[j];
                if (m == 0.0) continue;
                double vr = blk_re[i][j], vi = blk_im[i][j];
                if (PH) {
                    const double tr = vr * ph_c - vi * ph_s;
                    vi = fma(vr, ph_s, vi * ph_c);
                    vr = tr;
                }
                double *o = reinterpret_cast<double *>(prm.result) + 2 * (row * prm.ld + scol[j]);
                atomicAdd(o, vr * m);
                atomicAdd(o + 1, vi * m);
                if (SYM) {
                    double *ot = reinterpret_cast<double *>(prm.result) + 2 * (scol[j] * prm.ld + row);
                    atomicAdd(ot, vr * m);
                    atomicAdd(ot + 1, vi * m);
                }
            }
        }
    }
}

}  // namespace bc
