// Mixed-precision regular pairs of the single layer, double layer, adjoint
// double layer and hypersingular operators on P1 spaces (6-point rule) for the
// Helmholtz (Re k > 0, real or complex k), Laplace and modified Helmholtz
// kernels: the FP32 counterpart of regular_p1 (p1.cuh) with the geometry of
// the mixed DP0 kernels (dp0.cuh).
//
// Lengths are in units of 1/k.  Per element pair the centroid offset
// D = k (c_s - c_t), r_c' = |D| and exp(i r_c') are FP64; per point pair only
//   r'^2 - r_c'^2 = A_q + B_p + yo_q . m_p,
//   A_q = |yo_q|^2 + 2 D . yo_q,  B_p = |xo_p|^2 - 2 D . xo_p,  m_p = -2 xo_p,
// (xo, yo: the points' offsets from their centroids, times k) is formed in
// FP32, 1/r' by rsqrt.approx, the phase offset theta = (r'^2 - r_c'^2) /
// (r' + r_c') without cancellation and its sine / cosine by the fitted FP32
// polynomials; trial points q, q+1 travel together through packed f32x2 FMAs.
// Single layer: the trial sums T_j(p) = sum_q w_q psi_j(q) exp(i theta) / r'.
// Double layers: with h = (i r' - 1) exp(i theta) / r'^3 and d' = k (y - x),
// a quadrature point lies in its own element's plane, so
//   d' . n_s = D . n_s - xo_p . n_s      (one value per test point)
//   d' . n_t = D . n_t + yo_q . n_t      (one value per trial point);
// the double layer (trial normal) sums T_j(p) = sum_q w_q psi_j(q) h and
// multiplies by d'.n_s per test point, the adjoint double layer (test normal,
// kernel -(d . n_t)) sums h (-d'.n_t) per pair.  The 3 x 3 block
// sum_p w_p phi_i(p) T_j(p) is FP32 (36 terms per entry); it is converted to
// FP64 once per element pair, where k / (4 pi) (single layer, hypersingular)
// or k^2 / (4 pi) (double layers), the integration elements, exp(i r_c') and
// (hypersingular) the curl and normal products are applied.  SYM as in
// regular_p1: pairs i < j; single layer and hypersingular add the block at
// (i, j) and, unless deferred to the transpose pass, at (j, i); the double
// layers add at (j, i) the transposed pair's own block, which is the other
// operator's kernel of (i, j) (skew sweep: both normal sums per pair).
// Other kernels, in units of 1/kappa (kappa = Re k, omega, or 1 for Laplace):
// Laplace has no phase (1/r', -1/r'^3 in the double layers); modified
// Helmholtz exp(-r') = exp(-r_c') exp(-theta), the first FP64 per element
// pair, the second __expf per point pair, double-layer factor -(1 + r'); a
// complex wavenumber k = kr + i ki adds exp(-beta r'), beta = ki / kr, split
// the same way beside exp(i r'), the double-layer factor
// (i k r - 1) = -(1 + beta r') + i r', and -k^2 complex in the hypersingular
// operator.  Laplace and modified Helmholtz blocks are real and go to a real
// matrix.
// Maxwell magnetic field on RWG / SNC (ASM_MFIE): with u_i(p) = J_t r_i(p) =
// x_p - P_ti and v_j(q) = y_q - P_sj (P: the vertex each RWG function points
// away from), (x - y) . (u x v) = (P_ti - P_sj) . (u x v), so
//   MFIE_ij = sum_ab det(P_ti - P_sj, J_t^a, J_s^b) N_ab,
//   N_ab = sum_pq w_p w_q H (zeta_a(p) - o_ia)(zeta_b(q) - o_jb),
// zeta = (xi, eta), o_i = (a_i, b_i), H = e^{ikr} (ikr - 1) / r^3: the N are
// shifts of the nine moments of H, which the FP32 core gives as it gives
// the EFIE's moments of G (the double layer's kernel value h without its
// normal factor).  The determinants are FP64 geometry, so pairs of nearly
// coplanar elements, whose triple products nearly vanish, keep the FP32
// moments' relative accuracy (mfie_block_moments).
// Maxwell electric field on RWG / SNC (ASM_EFIE): the nine moments
// M[u][v] = sum_pq w_p w_q G u(p) v(q), u, v in {1, xi, eta}, that the EFIE
// block needs (rwg.cuh) are a fixed linear map of the P1 single-layer block
// (1 = phi_0 + phi_1 + phi_2, xi = phi_1, eta = phi_2), so the FP32 part is
// the single layer's and the FP64 epilogue forms the moments and
// efie_block; the integration elements cancel against the RWG basis.
// Scatter: the FP64 block entries of a warp's 32 pairs (one test element,
// 32 consecutive trial elements) are summed per distinct trial dof in shared
// memory and added to the matrix once per (test dof, trial dof)
// (warp_cols.cuh): ~3.5x fewer FP64 L2 atomics, which bound the double-layer
// sweep (each pair adds two blocks).
#pragma once

#include "p1.cuh"
#include "rwg.cuh"
#include "warp_cols.cuh"

namespace bc {

struct TestBlockP1m {
    float4 m[P1_TCHUNK][NQ6];  // (-2 xo, |xo|^2), xo = k (x_p - c_t)
    double c[P1_TCHUNK][3];
    double n[P1_TCHUNK][3];
    double ie[P1_TCHUNK];
    double mult[P1_TCHUNK][3];
    int64_t row[P1_TCHUNK][3];
    int v[P1_TCHUNK][3];
};

// NT, NS: test / trial functions per element, 3 (P1, DP1, RWG / SNC) or 1 (a P0 space beside a P1 one: its
// constant function takes the rule's weights in place of the P1 shape weights; scalar operators, no
// symmetric sweep).
template <int ASM, int K, int PHC, bool SYM, bool CK = false, int NT = 3, int NS = 3>
__global__ void __launch_bounds__(DP0_THREADS) regular_p1_mixed(RegParams prm, QuadRule rule) {
    constexpr bool LAP = K == BEMPPCUDA_LAPLACE_SLP || K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_LAPLACE_ADLP;
    constexpr bool MH = K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_MODHELM_ADLP;
    constexpr bool REAL = LAP || MH;  // real kernel, real result
    constexpr bool HYP = ASM == BEMPPCUDA_ASM_HELM_HYP || ASM == BEMPPCUDA_ASM_LAPLACE_HYP ||
                         ASM == BEMPPCUDA_ASM_MODHELM_HYP;
    constexpr bool EFIE = ASM == BEMPPCUDA_ASM_EFIE;  // test curl slots hold J_t, multipliers edge lengths
    constexpr bool MFIE = ASM == BEMPPCUDA_ASM_MFIE;  // the same, and v0_t in the third slot
    constexpr bool RWG = EFIE || MFIE;
    constexpr bool DL = K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_MODHELM_DLP;
    constexpr bool AD = K == BEMPPCUDA_HELMHOLTZ_ADLP || K == BEMPPCUDA_LAPLACE_ADLP || K == BEMPPCUDA_MODHELM_ADLP;
    static_assert(!CK || !REAL, "complex wavenumber: the Helmholtz kernels");
    static_assert((NT == 3 && NS == 3) || (ASM == BEMPPCUDA_ASM_SCALAR && !SYM && (NT == 1 || NS == 1)),
                  "P0 beside P1: scalar operators, per-pair sweep");
    constexpr bool SKEW = SYM && (DL || AD);
    constexpr bool NS_SUM = DL || SKEW;  // sums multiplied by d'.n_s per test point
    constexpr bool NT_SUM = AD || SKEW;  // sums with -d'.n_t per pair
    constexpr int NP = NQ6 / 2;
    __shared__ TestBlockP1m sb;
    __shared__ double scurl[HYP || RWG ? P1_TCHUNK : 1][3][3];  // curls (HYP) or J_t, v0_t (RWG)
    __shared__ WarpColumns swc[DP0_THREADS / 32];
    // staged block entries per warp: [block row][staging position]; SKEW: the (j, i) blocks too
    __shared__ double2 sst[DP0_THREADS / 32][3][WC_SLOTS];
    __shared__ double2 sst_t[SKEW ? DP0_THREADS / 32 : 1][3][SKEW ? WC_SLOTS : 1];
    // units of 1/kappa: kappa = k (Helmholtz; Re k for a complex wavenumber), omega (modified), 1 (Laplace)
    const double kap = LAP ? 1.0 : prm.p[0];
    // exp(-beta r') beside exp(i r'): beta = Im k / Re k (complex k), 1 (modified: exp(-r') alone)
    const double betd = CK ? prm.p[1] / prm.p[0] : (MH ? 1.0 : 0.0);
    const float bet = (float)betd;

    // test elements per CTA: P1_TCHUNK, and for the Maxwell operators ceil(ntest / gridDim.y) <= P1_TCHUNK
    // (their launch picks 16 on small grids; a runtime height made the scalar kernels slower)
    const int rows = RWG ? (int)((prm.ntest + gridDim.y - 1) / gridDim.y) : P1_TCHUNK;
    const int64_t t0 = (int64_t)blockIdx.y * rows;
    if (SYM && t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;  // below the diagonal
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
            sb.n[idx][d] = g.n[d];
            sb.v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            sb.mult[idx][i] = i < NT ? prm.tmult[t * NT + i] * (RWG ? edge_length(prm.tg, prm.tne, t, i) : 1.0) : 0.0;
            sb.row[idx][i] = i < NT ? prm.tl2g[t * NT + i] : 0;
        }
        if (RWG) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                scurl[idx][0][d] = g.j0[d];
                scurl[idx][1][d] = g.j1[d];
                scurl[idx][2][d] = g.v0[d];
            }
        }
        if (HYP) {
            double cu[3][3];
            surface_curls(prm.tg, prm.tne, t, g.n, cu);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int d = 0; d < 3; ++d) scurl[idx][i][d] = cu[i][d];
        }
        sb.ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    const bool active = si < prm.ntrial;  // lanes past the last trial element stage nothing
    if (__all_sync(0xffffffffu, !active)) return;
    const int64_t s = prm.ssup[active ? si : prm.ntrial - 1];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    double sc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sc[d] = __ldg(prm.sg + (22 + d) * prm.sne + s);
    // trial offsets k (y_q - c_s), q = 2 jj, 2 jj + 1 packed
    float2 yx[NP], yyy[NP], yz[NP], yy2[NP];
#pragma unroll
    for (int jj = 0; jj < NP; ++jj) {
        float o[2][3];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            double v[3];
            to_global(gs, rule.x[2 * jj + h], rule.y[2 * jj + h], v);
#pragma unroll
            for (int d = 0; d < 3; ++d) o[h][d] = (float)(kap * (v[d] - sc[d]));
        }
        yx[jj] = f2(o[0][0], o[1][0]);
        yyy[jj] = f2(o[0][1], o[1][1]);
        yz[jj] = f2(o[0][2], o[1][2]);
        yy2[jj] = fma2(yz[jj], yz[jj], fma2(yyy[jj], yyy[jj], mul2(yx[jj], yx[jj])));
    }
    const float sn0 = (float)gs.n[0], sn1 = (float)gs.n[1], sn2 = (float)gs.n[2];
    double curl_s[3][3];
    if (HYP) surface_curls(prm.sg, prm.sne, s, gs.n, curl_s);
    int64_t scol[3];
    double smul[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        scol[j] = j < NS ? prm.sl2g[s * NS + j] : -1;  // no slot past the element's functions
        smul[j] = j < NS ? prm.smult[s * NS + j] * (RWG ? edge_length(prm.sg, prm.sne, s, j) : 1.0) : 0.0;
    }
    // the warp's columns (distinct trial dofs) and this lane's staging positions
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    WarpColumns &wc = swc[warp];
    int pos[3];
    {
        int dof[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) dof[j] = active && scol[j] >= 0 && scol[j] < INT32_MAX ? (int)scol[j] : -1;
        static_assert(sizeof(sst[0]) >= 2 * WC_TABLE * sizeof(int), "column table scratch");
        wc_build(wc, reinterpret_cast<int *>(&sst[warp][0][0]), dof, pos);
    }
    double2(&st)[3][WC_SLOTS] = sst[warp];
    double2(&st_t)[3][SKEW ? WC_SLOTS : 1] = sst_t[SKEW ? warp : 0];

    for (int tt = 0; tt < tcount; ++tt) {
        const bool done = !active || (SYM && t0 + tt >= si);  // rows increase with tt
        if (__all_sync(0xffffffffu, done)) break;
        if (done || (prm.grids_identical && shares_vertex(sb.v[tt], sv0, sv1, sv2))) {
            // no pair: zeros in this lane's staging positions
#pragma unroll
            for (int i = 0; i < NT; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    if (pos[j] >= 0) {
                        st[i][pos[j]] = make_double2(0.0, 0.0);
                        if (SKEW) st_t[i][pos[j]] = make_double2(0.0, 0.0);
                    }
        } else {
        const double D0 = kap * (sc[0] - sb.c[tt][0]), D1 = kap * (sc[1] - sb.c[tt][1]),
                     D2 = kap * (sc[2] - sb.c[tt][2]);
        const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
        const double rc = sqrt(rc2);
        // the element pair's factor: exp(i r_c'), times exp(-beta r_c') (complex k); exp(-r_c') (modified)
        double ph_s = 0.0, ph_c = 1.0;
        if (!LAP) {
            if (!MH) sincos_cw64(rc, &ph_s, &ph_c);
            if (MH || CK) {
                const double am = exp(-betd * rc);
                ph_c *= am;
                ph_s *= am;
            }
        }
        const float D0f = (float)D0, D1f = (float)D1, D2f = (float)D2;
        const float2 rcf2 = b2((float)rc), rc2f2 = b2((float)rc2);
        const float2 D0d = b2(2.f * D0f), D1d = b2(2.f * D1f), D2d = b2(2.f * D2f);
        float2 A[NP];
#pragma unroll
        for (int jj = 0; jj < NP; ++jj) A[jj] = fma2(D2d, yz[jj], fma2(D1d, yyy[jj], fma2(D0d, yx[jj], yy2[jj])));
        // normal terms: D . n_s; -(d'.n_t) = -(D . n_t) - yo_q . n_t per trial point
        const float tn0 = (float)sb.n[tt][0], tn1 = (float)sb.n[tt][1], tn2 = (float)sb.n[tt][2];
        const float Dns = fmaf(D2f, sn2, fmaf(D1f, sn1, D0f * sn0));
        float2 mdt[NP];
        if (NT_SUM) {
            const float2 mDnt = b2(-fmaf(D2f, tn2, fmaf(D1f, tn1, D0f * tn0)));
#pragma unroll
            for (int jj = 0; jj < NP; ++jj)
                mdt[jj] = fma2(yz[jj], b2(-tn2), fma2(yyy[jj], b2(-tn1), fma2(yx[jj], b2(-tn0), mDnt)));
        }
        float lre[3][3], lim[3][3];              // block of (i, j): single layer, or the first double layer
        float ure[3][3], uim[3][3];              // SKEW: the transposed pair's block
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) lre[i][j] = lim[i][j] = ure[i][j] = uim[i][j] = 0.f;
#pragma unroll 2
        for (int p = 0; p < NQ6; ++p) {
            const float4 m = sb.m[tt][p];
            const float Bp = fmaf(D2f, m.z, fmaf(D1f, m.y, fmaf(D0f, m.x, m.w)));
            const float2 mx = b2(m.x), my = b2(m.y), mz = b2(m.z), Bp2 = b2(Bp);
            // d'.n_s at this test point: D . n_s - xo . n_s = D . n_s + (m . n_s) / 2
            const float dns = NS_SUM ? fmaf(0.5f, fmaf(m.z, sn2, fmaf(m.y, sn1, m.x * sn0)), Dns) : 0.f;
            float2 tre[3] = {b2(0.f), b2(0.f), b2(0.f)}, tim[3] = {b2(0.f), b2(0.f), b2(0.f)};
            float2 vre[3] = {b2(0.f), b2(0.f), b2(0.f)}, vim[3] = {b2(0.f), b2(0.f), b2(0.f)};
#pragma unroll
            for (int jj = 0; jj < NP; ++jj) {
                const float2 sdot = fma2(yz[jj], mz, fma2(yyy[jj], my, fma2(yx[jj], mx, add2(A[jj], Bp2))));
                const float2 r2 = add2(rc2f2, sdot);
                const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                // cs + i sn: exp(i theta) (Helmholtz), times exp(-beta theta) (complex k); exp(-theta)
                // (modified, sn = 0); 1 (Laplace)
                float2 sn = b2(0.f), cs = b2(1.f);
                if (!LAP) {
                    const float2 den = fma2(r2, rinv, rcf2);
                    const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                    if (!MH) sincos2<PHC>(th, &sn, &cs);
                    if (MH || CK) {
                        const float2 am = f2(__expf(-bet * th.x), __expf(-bet * th.y));
                        cs = mul2(cs, am);
                        if (CK) sn = mul2(sn, am);
                    }
                }
                float2 kr, ki = b2(0.f);
                if (!DL && !AD && !MFIE) {
                    kr = mul2(rinv, cs);
                    if (!REAL) ki = mul2(rinv, sn);
                } else if (LAP) {
                    kr = mul2(rinv, mul2(rinv, mul2(rinv, b2(-1.f))));  // -1 / r'^3
                } else {
                    // h = (i k r - 1) e^{ikr} / r^3 in units of 1/kappa: ((-a cs - r' sn) + i (r' cs - a sn)) / r'^3,
                    // a = 1 + beta r' (a = 1 for real k); modified: -(1 + r') e^{-r'} / r'^3
                    const float2 rp = mul2(r2, rinv), r3 = mul2(rinv, mul2(rinv, rinv));
                    if (MH) {
                        kr = mul2(mul2(r3, cs), mul2(add2(rp, b2(1.f)), b2(-1.f)));
                    } else if (CK) {
                        const float2 a = fma2(b2(bet), rp, b2(1.f));
                        kr = mul2(r3, mul2(fma2(rp, sn, mul2(a, cs)), b2(-1.f)));
                        ki = mul2(r3, fma2(rp, cs, mul2(mul2(a, sn), b2(-1.f))));
                    } else {
                        kr = mul2(r3, mul2(fma2(rp, sn, cs), b2(-1.f)));
                        ki = mul2(r3, fma2(rp, cs, mul2(sn, b2(-1.f))));
                    }
                }
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    const float2 w = NS == 3 ? f2(rule.swf[2 * jj][j], rule.swf[2 * jj + 1][j])
                                             : f2(rule.wf[2 * jj], rule.wf[2 * jj + 1]);
                    if (!AD || SKEW) {  // plain sums (single layer; double layer: times d'.n_s below)
                        tre[j] = fma2(kr, w, tre[j]);
                        if (!REAL) tim[j] = fma2(ki, w, tim[j]);
                    }
                    if (NT_SUM) {  // sums with -(d'.n_t)
                        const float2 wd = mul2(w, mdt[jj]);
                        vre[j] = fma2(kr, wd, vre[j]);
                        if (!REAL) vim[j] = fma2(ki, wd, vim[j]);
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < NT; ++i) {
                const float ph = NT == 3 ? rule.swf[p][i] : rule.wf[p];
                const float phs = NS_SUM ? ph * dns : ph;
#pragma unroll
                for (int j = 0; j < NS; ++j) {
                    if (!DL && !AD) {
                        lre[i][j] = fmaf(ph, tre[j].x + tre[j].y, lre[i][j]);
                        if (!REAL) lim[i][j] = fmaf(ph, tim[j].x + tim[j].y, lim[i][j]);
                    } else {
                        // (i, j): double layer -> n_s sums, adjoint -> n_t sums; SKEW: the other one at (j, i)
                        const float2 first_r = DL ? tre[j] : vre[j], first_i = DL ? tim[j] : vim[j];
                        const float f1 = DL ? phs : ph;
                        lre[i][j] = fmaf(f1, first_r.x + first_r.y, lre[i][j]);
                        if (!REAL) lim[i][j] = fmaf(f1, first_i.x + first_i.y, lim[i][j]);
                        if (SKEW) {
                            const float2 sec_r = DL ? vre[j] : tre[j], sec_i = DL ? vim[j] : tim[j];
                            const float f2_ = DL ? ph : phs;
                            ure[i][j] = fmaf(f2_, sec_r.x + sec_r.y, ure[i][j]);
                            if (!REAL) uim[i][j] = fmaf(f2_, sec_i.x + sec_i.y, uim[i][j]);
                        }
                    }
                }
            }
        }
        // k / (4 pi) or k^2 / (4 pi), |J_t| |J_s| exp(i r_c'), then the hypersingular combination;
        // EFIE: the moments, k (4 pi G = k e^{i theta} / r' in these units) and 1 / (4 pi), no |J|
        double ere[3][3], eim[3][3];
        if (EFIE) {
            double mre[3][3], mim[3][3];
            double rs[3] = {0.0, 0.0, 0.0}, is[3] = {0.0, 0.0, 0.0};  // sums over j (row sums)
            double cs_[3] = {0.0, 0.0, 0.0}, ci_[3] = {0.0, 0.0, 0.0};  // sums over i (column sums)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double lr = kap * (double)lre[i][j], li = kap * (double)lim[i][j];
                    rs[i] += lr;
                    is[i] += li;
                    cs_[j] += lr;
                    ci_[j] += li;
                }
            mre[0][0] = rs[0] + rs[1] + rs[2];
            mim[0][0] = is[0] + is[1] + is[2];
#pragma unroll
            for (int a = 1; a < 3; ++a) {
                mre[a][0] = rs[a];
                mim[a][0] = is[a];
                mre[0][a] = cs_[a];
                mim[0][a] = ci_[a];
#pragma unroll
                for (int b = 1; b < 3; ++b) {
                    mre[a][b] = kap * (double)lre[a][b];
                    mim[a][b] = kap * (double)lim[a][b];
                }
            }
            efie_block<CK>(mre, mim, scurl[tt][0], scurl[tt][1], gs.j0, gs.j1, kap, CK ? prm.p[1] : 0.0, ere, eim);
        } else if (MFIE) {
            // the moments of H = k^3 h (units of 1/k), then the block from the FP64 geometry
            const double k3 = kap * kap * kap;
            double mre[3][3], mim[3][3];
            double rs[3] = {0.0, 0.0, 0.0}, is[3] = {0.0, 0.0, 0.0};
            double cs_[3] = {0.0, 0.0, 0.0}, ci_[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const double lr = k3 * (double)lre[i][j], li = k3 * (double)lim[i][j];
                    rs[i] += lr;
                    is[i] += li;
                    cs_[j] += lr;
                    ci_[j] += li;
                    if (i > 0 && j > 0) {
                        mre[i][j] = lr;
                        mim[i][j] = li;
                    }
                }
            mre[0][0] = rs[0] + rs[1] + rs[2];
            mim[0][0] = is[0] + is[1] + is[2];
#pragma unroll
            for (int a = 1; a < 3; ++a) {
                mre[a][0] = rs[a];
                mim[a][0] = is[a];
                mre[0][a] = cs_[a];
                mim[0][a] = ci_[a];
            }
            mfie_block_moments(mre, mim, scurl[tt][2], scurl[tt][0], scurl[tt][1], gs.v0, gs.j0, gs.j1, ere, eim);
        }
        const double scale = RWG ? BC_INV_4PI : (DL || AD ? kap * kap : kap) * BC_INV_4PI * sb.ie[tt] * gs.ie;
        double sre = 0.0, sim = 0.0, cpf = 0.0, cpi = 0.0;
        if (HYP) {
            // S = sum_pq w_p w_q G: the P1 functions add up to 1 on each side
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    sre += (double)lre[i][j];
                    sim += (double)lim[i][j];
                }
            // -k^2 (n_t . n_s), complex for a complex wavenumber; +w^2 (n_t . n_s) modified; 0 Laplace
            const double nn = sb.n[tt][0] * gs.n[0] + sb.n[tt][1] * gs.n[1] + sb.n[tt][2] * gs.n[2];
            if (MH) {
                cpf = kap * kap * nn;
            } else if (!LAP) {
                const double ki = CK ? prm.p[1] : 0.0;
                cpf = -(kap * kap - ki * ki) * nn;
                cpi = -2.0 * kap * ki * nn;
            }
        }
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const double mt = sb.mult[tt][i];
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                const double ms = smul[j];
                if (pos[j] < 0) continue;
                if (mt == 0.0 || ms == 0.0) {
                    st[i][pos[j]] = make_double2(0.0, 0.0);
                    if (SKEW) st_t[i][pos[j]] = make_double2(0.0, 0.0);
                    continue;
                }
                double vr = RWG ? ere[i][j] : (double)lre[i][j], vi = RWG ? eim[i][j] : (double)lim[i][j];
                if (HYP) {
                    const double cij = scurl[tt][i][0] * curl_s[j][0] + scurl[tt][i][1] * curl_s[j][1] +
                                       scurl[tt][i][2] * curl_s[j][2];
                    const double lr = vr, li = vi;
                    vr = fma(cij, sre, fma(cpf, lr, -cpi * li));
                    vi = fma(cij, sim, fma(cpf, li, cpi * lr));
                }
                const double tr = vr * ph_c - vi * ph_s;
                vi = fma(vr, ph_s, vi * ph_c);
                vr = tr;
                double wr = vr, wi = vi;  // the (j, i) block: the same, or (SKEW) its own sums
                if (SKEW) {
                    const double ur = (double)ure[i][j], ui = (double)uim[i][j];
                    wr = ur * ph_c - ui * ph_s;
                    wi = fma(ur, ph_s, ui * ph_c);
                }
                const double mm = mt * ms * scale;
                st[i][pos[j]] = make_double2(vr * mm, vi * mm);
                if (SKEW) st_t[i][pos[j]] = make_double2(wr * mm, wi * mm);
            }
        }
        }  // pair
        __syncwarp();
        // per (test dof, column): the sum of the column's staged entries, one complex atomic
        // (and, for the symmetric sweep, one at the transposed position)
        const int ncols = wc.ncols;
        double *res = reinterpret_cast<double *>(prm.result);
        // one entry into the matrix: complex (two atomics) or, for the real kernels, real
        const auto add_entry = [](double *m, int64_t ld, int64_t r, int64_t c, double re, double im) {
            if (REAL) {
                atomicAdd(m + r * ld + c, re);
            } else {
                atomicAdd(m + 2 * (r * ld + c), re);
                atomicAdd(m + 2 * (r * ld + c) + 1, im);
            }
        };
#pragma unroll
        for (int i = 0; i < NT; ++i) {
            const int64_t row = sb.row[tt][i];
            for (int c = (int)lane; c < ncols; c += 32) {
                const int b = wc.start[c], e = wc.start[c + 1];
                double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
                for (int k = b; k < e; ++k) {
                    const double2 v = st[i][k];
                    ar += v.x;
                    ai += v.y;
                    if (SKEW) {
                        const double2 w = st_t[i][k];
                        br += w.x;
                        bi += w.y;
                    }
                }
                const int64_t col = wc.col[c];
                if (ar != 0.0 || ai != 0.0) {
                    add_entry(res, prm.ld, row, col, ar, ai);
                    if (SYM && !SKEW && !prm.defer_transpose) add_entry(res, prm.ld, col, row, ar, ai);
                }
                if (SKEW && (br != 0.0 || bi != 0.0)) add_entry(res, prm.ld, col, row, br, bi);
            }
        }
        __syncwarp();  // the staging arrays are rewritten by the next test element
    }
}

}  // namespace bc
