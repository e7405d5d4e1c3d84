// Singular (adjacent) pairs of the Maxwell electric and magnetic field
// operators on RWG / SNC: maxwell_efield_singular and maxwell_mfield_singular
// (numba_kernels.py:1973-2147) for the dense and per-pair outputs, in place of
// the generic singular_pairs kernel.
//
// One warp per pair, the lanes over its Sauter-Schwab points, summing what
// the regular kernels sum per element pair (rwg.cuh): the nine moments
// M[a][b] = sum w G u_a(x) v_b(y), u, v = (1, xi, eta) for the electric field,
// and the four sums PB, PC, QB, QC of H = w G (ikr - 1) / r^2 for the magnetic
// field; efie_block / mfie_block turn them into the 3 x 3 block.  As in
// singular_p1, for a real wavenumber exp(ikr) is factored about the centroid
// distance r_c (|r - r_c| <= R_t + R_s for adjacent pairs; phase classes 1, 2,
// one rotation by exp(i k r_c) per pair), the lane sums are reduced through a
// shared table in a fixed order, and the block entries are finished by nine
// lanes at once (one entry and its atomic adds each) instead of one lane.
#pragma once

#include "common.cuh"
#include "rwg.cuh"

namespace bc {

template <int ASM, int PHC>
__global__ void __launch_bounds__(32 * SING_WARPS) singular_rwg(SingParams prm) {
    constexpr bool MFIE = ASM == BEMPPCUDA_ASM_MFIE;
    static_assert(MFIE || ASM == BEMPPCUDA_ASM_EFIE, "Maxwell operators");
    constexpr bool PH = PHC == 1 || PHC == 2;
    constexpr bool CK = PHC == 3;
    // EFIE: M[a][b] re / im at 2 (3 a + b); MFIE: PB (0, 1), PC (2 + 2c, 3 + 2c), QB (8 + ..), QC (14 + ..)
    constexpr int NV = MFIE ? 20 : 18;
    __shared__ double red[SING_WARPS][NV][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t k = (int64_t)blockIdx.x * SING_WARPS + warp;
    if (k >= prm.npairs || !pair_in_range(prm, k)) return;
    const int64_t t = prm.te[k], s = prm.se[k];
    Geom gt, gs;
    load_geom(prm.g, prm.ne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
    load_geom(prm.g, prm.ne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const double kr = prm.p[0], ki = CK ? prm.p[1] : 0.0;
    double rc = 0.0;
    if (PH) {
        const double D0 = __ldg(prm.g + 22 * prm.ne + s) - __ldg(prm.g + 22 * prm.ne + t);
        const double D1 = __ldg(prm.g + 23 * prm.ne + s) - __ldg(prm.g + 23 * prm.ne + t);
        const double D2 = __ldg(prm.g + 24 * prm.ne + s) - __ldg(prm.g + 24 * prm.ne + t);
        rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
    }
    double v[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = 0.0;

    const int64_t toff = prm.toff[k], soff = prm.soff[k], woff = prm.woff[k];
    const int n = (int)prm.npts[k];
    for (int m = lane; m < n; m += 32) {
        const double2 tpm = reinterpret_cast<const double2 *>(prm.tp)[toff + m];
        const double2 spm = reinterpret_cast<const double2 *>(prm.sp)[soff + m];
        const double w = __ldg(prm.w + woff + m);
        double x[3], y[3];
        to_global(gt, tpm.x, tpm.y, x);
        to_global(gs, spm.x, spm.y, y);
        const double df[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
        const double r2 = fma(df[2], df[2], fma(df[1], df[1], df[0] * df[0]));
        const double rinv = rsqrt64(r2);
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
        // w G without 1 / (4 pi) and the pair's phase factor exp(i k r_c)
        const double gw = w * rinv, kwr = gw * cs, kwi = gw * sn;
        if (!MFIE) {
            const double ut[3] = {1.0, tpm.x, tpm.y}, vs[3] = {1.0, spm.x, spm.y};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double wr = kwr * ut[a], wi = kwi * ut[a];
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    v[2 * (3 * a + b)] = fma(wr, vs[b], v[2 * (3 * a + b)]);
                    v[2 * (3 * a + b) + 1] = fma(wi, vs[b], v[2 * (3 * a + b) + 1]);
                }
            }
        } else {
            // H = w G (ikr - 1) / r^2, (ikr - 1) = -(1 + ki r) + i kr r
            const double a = -fma(ki, r, 1.0) * rinv * rinv, b = kr * rinv;
            const double fr = kwr * a - kwi * b, fi = fma(kwr, b, kwi * a);
            double wt[3], ws[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                wt[c] = fma(gt.j1[c], tpm.y, gt.j0[c] * tpm.x);
                ws[c] = fma(gs.j1[c], spm.y, gs.j0[c] * spm.x);
            }
            const double wxd[3] = {fma(ws[1], df[2], -ws[2] * df[1]), fma(ws[2], df[0], -ws[0] * df[2]),
                                   fma(ws[0], df[1], -ws[1] * df[0])};
            const double dxw[3] = {fma(df[1], wt[2], -df[2] * wt[1]), fma(df[2], wt[0], -df[0] * wt[2]),
                                   fma(df[0], wt[1], -df[1] * wt[0])};
            const double pb = fma(wt[2], wxd[2], fma(wt[1], wxd[1], wt[0] * wxd[0]));
            v[0] = fma(fr, pb, v[0]);
            v[1] = fma(fi, pb, v[1]);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                v[2 + 2 * c] = fma(fr, dxw[c], v[2 + 2 * c]);
                v[3 + 2 * c] = fma(fi, dxw[c], v[3 + 2 * c]);
                v[8 + 2 * c] = fma(fr, wxd[c], v[8 + 2 * c]);
                v[9 + 2 * c] = fma(fi, wxd[c], v[9 + 2 * c]);
                v[14 + 2 * c] = fma(fr, df[c], v[14 + 2 * c]);
                v[15 + 2 * c] = fma(fi, df[c], v[15 + 2 * c]);
            }
        }
    }

    // lane l < NV sums value l over the 32 lanes (row l, in lane order) into column 32 of its row;
    // every lane then reads all totals
#pragma unroll
    for (int i = 0; i < NV; ++i) red[warp][i][lane] = v[i];
    __syncwarp();
    if (lane < NV) {
        double tot = 0.0;
#pragma unroll 8
        for (int m = 0; m < 32; ++m) tot += red[warp][lane][m];
        red[warp][lane][32] = tot;
    }
    __syncwarp();
    if (lane >= 9) return;
    double ph_s = 0.0, ph_c = 1.0;
    if (PH) sincos_cw64(kr * rc, &ph_s, &ph_c);
#pragma unroll
    for (int i = 0; i < NV / 2; ++i) {
        const double a = red[warp][2 * i][32], b = red[warp][2 * i + 1][32];
        v[2 * i] = PH ? a * ph_c - b * ph_s : a;
        v[2 * i + 1] = PH ? fma(a, ph_s, b * ph_c) : b;
    }
    double blk_re[3][3], blk_im[3][3];
    if (!MFIE) {
        double mre[3][3], mim[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                mre[a][b] = v[2 * (3 * a + b)];
                mim[a][b] = v[2 * (3 * a + b) + 1];
            }
        efie_block<CK>(mre, mim, gt.j0, gt.j1, gs.j0, gs.j1, kr, ki, blk_re, blk_im);
    } else {
        const double pcr[3] = {v[2], v[4], v[6]}, pci[3] = {v[3], v[5], v[7]};
        const double qbr[3] = {v[8], v[10], v[12]}, qbi[3] = {v[9], v[11], v[13]};
        const double qcr[3] = {v[14], v[16], v[18]}, qci[3] = {v[15], v[17], v[19]};
        mfie_block(v[0], v[1], pcr, pci, qbr, qbi, qcr, qci, gt.j0, gt.j1, gs.j0, gs.j1, blk_re, blk_im);
    }
    // this lane's entry (i, j) = (lane / 3, lane % 3), selected with compile-time indexes
    const int i = lane / 3, j = lane - 3 * (lane / 3);
    double er = 0.0, ei = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
            if (a == i && b == j) {
                er = blk_re[a][b];
                ei = blk_im[a][b];
            }
    // the |J| factors cancel in the RWG functions; the two edge lengths remain
    const double f = BC_INV_4PI * edge_length(prm.g, prm.ne, t, i) * edge_length(prm.g, prm.ne, s, j);
    const double vr = er * f, vi = ei * f;
    if (prm.values) {
        const int64_t idx = (k * 3 + i) * 3 + j;
        if (prm.is_complex) {
            double *o = reinterpret_cast<double *>(prm.values) + 2 * idx;
            o[0] += vr;
            o[1] += vi;
        } else {
            reinterpret_cast<double *>(prm.values)[idx] += vr;
        }
        return;
    }
    const double mt = prm.tmult[t * 3 + i], ms = prm.smult[s * 3 + j];
    if (mt == 0.0 || ms == 0.0) return;
    const int64_t row = prm.tl2g[t * 3 + i], col = prm.sl2g[s * 3 + j];
    const double mm = mt * ms;
    if (prm.is_complex) {
        double *o = reinterpret_cast<double *>(prm.dense) + 2 * (row * prm.ld + col);
        atomicAdd(o, vr * mm);
        atomicAdd(o + 1, vi * mm);
    } else {
        atomicAdd(reinterpret_cast<double *>(prm.dense) + row * prm.ld + col, vr * mm);
    }
}

}  // namespace bc
