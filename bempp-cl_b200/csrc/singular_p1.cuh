// Singular (adjacent) pairs of the scalar kernels and the hypersingular
// operators on P1 x P1 (three shape functions on both elements): the kernels
// of default_scalar_singular_kernel (numba_kernels.py:1471-1526) and
// laplace/helmholtz/modified hypersingular_singular (:1530-1784) restricted to
// linear shapes, where the generic singular_pairs kernel carries runtime shape
// counts.
//
// One warp per pair, the lanes over its Sauter-Schwab points as in
// singular_pairs, with three differences:
// * shapes known at compile time (phi = 1 - u - v, u, v);
// * for a real wavenumber exp(ikr) is factored about the centroid distance
//   r_c as in the DP0 singular kernel (|r - r_c| <= R_t + R_s also for
//   adjacent pairs), so the per-point phase is a short polynomial (phase
//   classes 1 and 2) and the block is rotated by exp(i k r_c) once;
// * the warp's partial sums go through shared memory (lane v sums row v of a
//   values x 32 table in a fixed order) instead of one shuffle tree per value,
//   and each lane then owns one block entry and issues its own atomic adds.
// A vertex-adjacent pair of one space in dense mode (the rule lists the pair
// in both orders with the points exchanged) gives both blocks for the kernels
// symmetric in x and y (single layers and hypersingular operators: the block
// of (s, t) is the transpose of that of (t, s)), evaluated at the pair with
// t < s; the double layers evaluate both orders.
#pragma once

#include "common.cuh"
#include "singular_dp0.cuh"

namespace bc {

template <int ASM, int K, int PHC>
struct SingP1Traits {
    using T = SingDp0Traits<K>;
    static constexpr bool lhyp = ASM == BEMPPCUDA_ASM_LAPLACE_HYP;
    static constexpr bool hyp = lhyp || ASM == BEMPPCUDA_ASM_HELM_HYP || ASM == BEMPPCUDA_ASM_MODHELM_HYP;
    static constexpr bool helm = T::helm;
    static constexpr bool ph = helm && (PHC == 1 || PHC == 2);  // centroid-factored phase
    static constexpr bool ck = helm && PHC == 3;                // complex wavenumber
    static constexpr bool dla = T::dl || T::ad;                 // double-layer family
    static constexpr int nc = helm ? 2 : 1;                     // doubles per value
    static constexpr int nblock = lhyp ? 0 : 9;                 // block entries summed
    static constexpr int nsum = hyp ? 1 : 0;                    // S = sum_p w G (hypersingular)
    static constexpr int nv = (nblock + nsum) * nc;             // doubles reduced per pair
    static constexpr bool symmetric = !dla;                     // G(x, y) = G(y, x)
    static_assert(nv <= 32, "one value per lane");
};

template <int ASM, int K, int PHC>
__global__ void __launch_bounds__(32 * SING_WARPS) singular_p1(SingParams prm) {
    using S = SingP1Traits<ASM, K, PHC>;
    constexpr int NV = S::nv;
    __shared__ double red[SING_WARPS][NV][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t k = (int64_t)blockIdx.x * SING_WARPS + warp;
    if (k >= prm.npairs || !pair_in_range(prm, k)) return;
    const int64_t t = prm.te[k], s = prm.se[k];
    const bool mirror = S::symmetric && !prm.values && prm.mirror_woff > 0 && (int64_t)prm.woff[k] == prm.mirror_woff;
    if (mirror && t > s) return;
    Geom gt, gs;
    load_geom(prm.g, prm.ne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
    load_geom(prm.g, prm.ne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const double kr = prm.p[0], ki = S::ck ? prm.p[1] : 0.0;
    double rc = 0.0;
    if (S::ph) {
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
        const double d0 = y[0] - x[0], d1 = y[1] - x[1], d2 = y[2] - x[2];
        const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
        const double rinv = rsqrt64(r2);
        const double r = r2 * rinv;
        // g: w times the kernel without 1 / (4 pi); the double layers' radial factor
        // rho_DL = (ikr - 1) e^{ikr} / r^3 (Laplace -1 / r^3, modified Helmholtz -(1 + w r) e^{-w r} / r^3)
        // times the normal term, (y - x).n_s for the double layer, -(y - x).n_t for the adjoint
        double gre, gim = 0.0;
        if (S::helm) {
            double sn, cs;
            if (S::ph && PHC == 2)
                sincos_half64(kr * (r - rc), &sn, &cs);
            else if (S::ph)
                sincos_small64(kr * (r - rc), &sn, &cs);
            else
                sincos_cw64(kr * r, &sn, &cs);
            if (S::ck) {
                const double am = exp(-ki * r);
                sn *= am;
                cs *= am;
            }
            if (!S::dla) {
                const double f = w * rinv;
                gre = f * cs;
                gim = f * sn;
            } else {
                const double q = w * rinv * rinv * rinv, a = -fma(ki, r, 1.0), b = kr * r;
                gre = q * fma(a, cs, -b * sn);
                gim = q * fma(b, cs, a * sn);
            }
        } else if (S::T::mh) {
            const double e = exp(-kr * r);
            gre = S::dla ? -w * fma(kr, r, 1.0) * e * rinv * rinv * rinv : w * e * rinv;
        } else {
            gre = S::dla ? -w * rinv * rinv * rinv : w * rinv;
        }
        if (S::dla) {
            const double dn = S::T::dl ? fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]))
                                       : -fma(d2, gt.n[2], fma(d1, gt.n[1], d0 * gt.n[0]));
            gre *= dn;
            gim *= dn;
        }
        if (S::nblock) {
            const double pt[3] = {1.0 - tpm.x - tpm.y, tpm.x, tpm.y};
            const double ps[3] = {1.0 - spm.x - spm.y, spm.x, spm.y};
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double ar = gre * pt[i], ai = gim * pt[i];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    v[(3 * i + j) * S::nc] = fma(ar, ps[j], v[(3 * i + j) * S::nc]);
                    if (S::helm) v[(3 * i + j) * S::nc + S::nc - 1] = fma(ai, ps[j], v[(3 * i + j) * S::nc + S::nc - 1]);
                }
            }
        }
        if (S::nsum) {
            v[S::nblock * S::nc] += gre;
            if (S::helm) v[S::nblock * S::nc + S::nc - 1] += gim;
        }
    }

    // lane l < NV sums value l over the 32 lanes (row l of the table, in lane order)
#pragma unroll
    for (int i = 0; i < NV; ++i) red[warp][i][lane] = v[i];
    __syncwarp();
    double tot = 0.0;
    if (lane < NV) {
#pragma unroll 8
        for (int m = 0; m < 32; ++m) tot += red[warp][lane][m];
    }
    // complex values: the imaginary part comes from the next lane
    const double tim = S::helm ? __shfl_down_sync(0xffffffffu, tot, 1) : 0.0;
    double sre = 0.0, sim = 0.0;  // S of the hypersingular operators, in every lane
    if (S::nsum) {
        sre = __shfl_sync(0xffffffffu, tot, S::nblock * S::nc);
        if (S::helm) sim = __shfl_sync(0xffffffffu, tot, S::nblock * S::nc + 1);
    }
    const int e = S::lhyp ? lane : lane / S::nc;  // the block entry this lane writes
    if (e >= 9 || (S::helm && !S::lhyp && (lane & 1))) return;
    const int i = e / 3, j = e - 3 * i;
    double mre = S::lhyp ? 0.0 : tot, mim = S::lhyp ? 0.0 : tim;
    if (S::ph) {
        double ps_, pc_;
        sincos_cw64(kr * rc, &ps_, &pc_);
        const double a = mre * pc_ - mim * ps_, b = fma(mre, ps_, mim * pc_);
        mre = a;
        mim = b;
        if (S::nsum) {
            const double c = sre * pc_ - sim * ps_, d = fma(sre, ps_, sim * pc_);
            sre = c;
            sim = d;
        }
    }
    const double scale = BC_INV_4PI * gt.ie * gs.ie;
    double vr, vi;
    if (S::hyp) {
        double ct[3][3], cs[3][3], cti[3], csj[3];
        surface_curls(prm.g, prm.ne, t, gt.n, ct);
        surface_curls(prm.g, prm.ne, s, gs.n, cs);
        // rows i and j by selection (lane-dependent indexes into register arrays would go to the stack)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            cti[d] = i == 0 ? ct[0][d] : (i == 1 ? ct[1][d] : ct[2][d]);
            csj[d] = j == 0 ? cs[0][d] : (j == 1 ? cs[1][d] : cs[2][d]);
        }
        const double cp = cti[0] * csj[0] + cti[1] * csj[1] + cti[2] * csj[2];
        if (S::lhyp) {
            vr = sre * scale * cp;
            vi = 0.0;
        } else {
            // c = -k^2 (Helmholtz, complex k allowed) or +omega^2 (modified Helmholtz)
            const double k2r = S::helm ? -(kr * kr - ki * ki) : kr * kr;
            const double k2i = S::helm ? -(2.0 * kr * ki) : 0.0;
            const double np = gt.n[0] * gs.n[0] + gt.n[1] * gs.n[1] + gt.n[2] * gs.n[2];
            const double mr = mre * np, mi = mim * np;
            vr = fma(cp, sre, fma(k2r, mr, -k2i * mi)) * scale;
            vi = fma(cp, sim, fma(k2r, mi, k2i * mr)) * scale;
        }
    } else {
        vr = mre * scale;
        vi = mim * scale;
    }
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
    const auto scatter = [&](int64_t te_, int ti, int64_t se_, int sj) {
        const double mt = prm.tmult[te_ * 3 + ti], ms = prm.smult[se_ * 3 + sj];
        if (mt == 0.0 || ms == 0.0) return;
        const int64_t row = prm.tl2g[te_ * 3 + ti], col = prm.sl2g[se_ * 3 + sj];
        const double mm = mt * ms;
        if (prm.is_complex) {
            double *o = reinterpret_cast<double *>(prm.dense) + 2 * (row * prm.ld + col);
            atomicAdd(o, vr * mm);
            atomicAdd(o + 1, vi * mm);
        } else {
            atomicAdd(reinterpret_cast<double *>(prm.dense) + row * prm.ld + col, vr * mm);
        }
    };
    scatter(t, i, s, j);
    if (mirror) scatter(s, j, t, i);  // the (s, t) block is the transpose
}

}  // namespace bc
