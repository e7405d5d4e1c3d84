// Singular (adjacent) DP0 pairs of the scalar kernels: the 3 x 3 local block
// reduces to one value, and for a real wavenumber exp(ikr) is factored about
// the centroid distance r_c as in the regular DP0 kernels: for any x in
// element i and y in element j, |r - r_c| <= R_i + R_j, so phase class PHC
// (|k|(R_i + R_j) <= 1 or 1/2) bounds the per-point phase offset for adjacent
// pairs as well.  PHC 3 is a complex wavenumber k = kr + i ki (exp(i kr r)
// exp(-ki r) per point, (ikr - 1) / r = -(1/r + ki) + i kr); modified
// Helmholtz (real, w = p[0]) scales the Laplace sums by exp(-w r) or
// exp(-w r) (1 + w r).  One warp per pair, lanes over the points.
// Used by the single-problem singular kernel and the batched one.
#pragma once

#include "common.cuh"

namespace bc {

template <int K>
struct SingDp0Traits {
    static constexpr bool helm = (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                                  K == BEMPPCUDA_HELMHOLTZ_ADLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool mh = (K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP ||
                                K == BEMPPCUDA_MODHELM_ADLP);
    static constexpr bool sl = (K == BEMPPCUDA_LAPLACE_SLP || K == BEMPPCUDA_HELMHOLTZ_SLP ||
                                K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool dl = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                                K == BEMPPCUDA_MODHELM_DLP || K == BEMPPCUDA_HELMHOLTZ_COMBINED);
    static constexpr bool ad = (K == BEMPPCUDA_LAPLACE_ADLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
                                K == BEMPPCUDA_MODHELM_ADLP);
};

// exp(-w r) for the single layer, exp(-w r) (1 + w r) for the double layers (modified Helmholtz)
__device__ __forceinline__ void mh_factors(double w, double r, double *e, double *e1) {
    *e = exp(-w * r);
    *e1 = *e * fma(w, r, 1.0);
}

// Kernel sum of one adjacent pair over its Sauter-Schwab points, without the
// integration elements and 1/(4 pi); every lane returns the warp total.
// g: geometry record (for the centroids), t / s: the pair, p: kernel parameters.
template <int K, int PHC>
__device__ __forceinline__ void sing_dp0_value(const double *__restrict__ g, int64_t ne, int64_t t, int64_t s,
                                               const Geom &gt, const Geom &gs, const double *p,
                                               const double2 *__restrict__ tp, const double2 *__restrict__ sp,
                                               const double *__restrict__ w, int64_t toff, int64_t soff,
                                               int64_t woff, int n, double *vr_out, double *vi_out) {
    using T = SingDp0Traits<K>;
    constexpr bool PH = T::helm && (PHC == 1 || PHC == 2);
    constexpr bool CK = T::helm && PHC == 3;
    const int lane = threadIdx.x & 31;
    const double kr = p[0], ki = CK ? p[1] : 0.0;
    double rc = 0.0;
    if (PH) {
        const double D0 = __ldg(g + 22 * ne + s) - __ldg(g + 22 * ne + t);
        const double D1 = __ldg(g + 23 * ne + s) - __ldg(g + 23 * ne + t);
        const double D2 = __ldg(g + 24 * ne + s) - __ldg(g + 24 * ne + t);
        rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
    }
    const double *nv = T::ad ? gt.n : gs.n;
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0;
    for (int m = lane; m < n; m += 32) {
        const double2 tpm = tp[toff + m];
        const double2 spm = sp[soff + m];
        const double wm = __ldg(w + woff + m);
        double x[3], y[3];
        to_global(gt, tpm.x, tpm.y, x);
        to_global(gs, spm.x, spm.y, y);
        const double d0 = y[0] - x[0], d1 = y[1] - x[1], d2 = y[2] - x[2];
        const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
        const double rinv = rsqrt64(r2);
        const double f = wm * rinv;
        double dot = 0.0;
        if (T::dl || T::ad) dot = (T::ad ? -1.0 : 1.0) * fma(d2, nv[2], fma(d1, nv[1], d0 * nv[0]));
        if (!T::helm) {
            double e = 1.0, e1 = 1.0;
            if (T::mh) mh_factors(kr, r2 * rinv, &e, &e1);
            if (T::sl) s0r = T::mh ? fma(f, e, s0r) : s0r + f;
            if (T::dl || T::ad) s1r = fma(f * dot * (T::mh ? e1 : 1.0), rinv * rinv, s1r);
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
            if (T::sl) {
                s0r = fma(f, cs, s0r);
                s0i = fma(f, sn, s0i);
            }
            if (T::dl || T::ad) {
                // (ikr - 1) e^{ikr} (dot) / r^3 = g (-h1 + i h2), g = f dot / r
                const double gg = f * dot * rinv, rk = rinv + ki;
                s1r = fma(gg, fma(rk, cs, kr * sn), s1r);
                s1i = fma(gg, fma(kr, cs, -rk * sn), s1i);
            }
        }
    }
    s0r = warp_sum(s0r);
    if (T::helm) s0i = warp_sum(s0i);
    if (T::dl || T::ad) {
        s1r = warp_sum(s1r);
        if (T::helm) s1i = warp_sum(s1i);
    }
    // SLP s0; Laplace DLP -s1r; Helmholtz DLP -s1r + i s1i; combined eta s0 + DLP
    double vr = 0.0, vi = 0.0;
    if (T::sl && K != BEMPPCUDA_HELMHOLTZ_COMBINED) {
        vr = s0r;
        vi = s0i;
    } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
        vr = fma(p[2], s0r, fma(-p[3], s0i, -s1r));
        vi = fma(p[2], s0i, fma(p[3], s0r, s1i));
    } else {
        vr = -s1r;
        vi = T::helm ? s1i : 0.0;
    }
    if (PH) {
        double ps, pc;
        sincos_cw64(kr * rc, &ps, &pc);
        const double tr = vr * pc - vi * ps;
        vi = fma(vr, ps, vi * pc);
        vr = tr;
    }
    *vr_out = vr;
    *vi_out = vi;
}

// Both orders of an adjacent pair whose reverse uses the same points with the
// roles exchanged (the vertex-adjacent rule): (vr, vi) for test t / trial s,
// (ur, ui) for test s / trial t.  The single layer is shared; the double
// layer of (s, t) takes the normal of t and d' = -d, the adjoint double layer
// the normal of s.
template <int K, int PHC>
__device__ __forceinline__ void sing_dp0_pair(const double *__restrict__ g, int64_t ne, int64_t t, int64_t s,
                                              const Geom &gt, const Geom &gs, const double *p,
                                              const double2 *__restrict__ tp, const double2 *__restrict__ sp,
                                              const double *__restrict__ w, int64_t toff, int64_t soff,
                                              int64_t woff, int n, double *vr_out, double *vi_out,
                                              double *ur_out, double *ui_out) {
    using T = SingDp0Traits<K>;
    constexpr bool PH = T::helm && (PHC == 1 || PHC == 2);
    constexpr bool CK = T::helm && PHC == 3;
    constexpr bool NORMAL = T::dl || T::ad;
    const int lane = threadIdx.x & 31;
    const double kr = p[0], ki = CK ? p[1] : 0.0;
    double rc = 0.0;
    if (PH) {
        const double D0 = __ldg(g + 22 * ne + s) - __ldg(g + 22 * ne + t);
        const double D1 = __ldg(g + 23 * ne + s) - __ldg(g + 23 * ne + t);
        const double D2 = __ldg(g + 24 * ne + s) - __ldg(g + 24 * ne + t);
        rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
    }
    // s0: single layer (both orders); s1: normal term of (t, s); s2: of (s, t)
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0, s2r = 0.0, s2i = 0.0;
    for (int m = lane; m < n; m += 32) {
        const double2 tpm = tp[toff + m];
        const double2 spm = sp[soff + m];
        const double wm = __ldg(w + woff + m);
        double x[3], y[3];
        to_global(gt, tpm.x, tpm.y, x);
        to_global(gs, spm.x, spm.y, y);
        const double d0 = y[0] - x[0], d1 = y[1] - x[1], d2 = y[2] - x[2];
        const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
        const double rinv = rsqrt64(r2);
        const double f = wm * rinv;
        double dot1 = 0.0, dot2 = 0.0;
        if (NORMAL) {
            const double dns = fma(d2, gs.n[2], fma(d1, gs.n[1], d0 * gs.n[0]));
            const double dnt = fma(d2, gt.n[2], fma(d1, gt.n[1], d0 * gt.n[0]));
            // double layer: (t, s) (y - x).n_s, (s, t) (x - y).n_t; adjoint: -(y - x).n_t, -(x - y).n_s
            dot1 = T::ad ? -dnt : dns;
            dot2 = T::ad ? dns : -dnt;
        }
        if (!T::helm) {
            double e = 1.0, e1 = 1.0;
            if (T::mh) mh_factors(kr, r2 * rinv, &e, &e1);
            if (T::sl) s0r = T::mh ? fma(f, e, s0r) : s0r + f;
            if (NORMAL) {
                const double f3 = f * rinv * rinv * (T::mh ? e1 : 1.0);
                s1r = fma(f3, dot1, s1r);
                s2r = fma(f3, dot2, s2r);
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
            if (T::sl) {
                s0r = fma(f, cs, s0r);
                s0i = fma(f, sn, s0i);
            }
            if (NORMAL) {
                const double fr = f * rinv, rk = rinv + ki;
                const double h1 = fma(rk, cs, kr * sn), h2 = fma(kr, cs, -rk * sn);
                const double g1 = fr * dot1, g2 = fr * dot2;
                s1r = fma(g1, h1, s1r);
                s1i = fma(g1, h2, s1i);
                s2r = fma(g2, h1, s2r);
                s2i = fma(g2, h2, s2i);
            }
        }
    }
    s0r = warp_sum(s0r);
    if (T::helm) s0i = warp_sum(s0i);
    if (NORMAL) {
        s1r = warp_sum(s1r);
        s2r = warp_sum(s2r);
        if (T::helm) {
            s1i = warp_sum(s1i);
            s2i = warp_sum(s2i);
        }
    }
    double v[2][2];
    const double nr[2] = {s1r, s2r}, ni[2] = {s1i, s2i};
#pragma unroll
    for (int o = 0; o < 2; ++o) {
        double vr = 0.0, vi = 0.0;
        if (T::sl && K != BEMPPCUDA_HELMHOLTZ_COMBINED) {
            vr = s0r;
            vi = s0i;
        } else if (K == BEMPPCUDA_HELMHOLTZ_COMBINED) {
            vr = fma(p[2], s0r, fma(-p[3], s0i, -nr[o]));
            vi = fma(p[2], s0i, fma(p[3], s0r, ni[o]));
        } else {
            vr = -nr[o];
            vi = T::helm ? ni[o] : 0.0;
        }
        if (PH) {
            double ps, pc;
            sincos_cw64(kr * rc, &ps, &pc);
            const double tr = vr * pc - vi * ps;
            vi = fma(vr, ps, vi * pc);
            vr = tr;
        }
        v[o][0] = vr;
        v[o][1] = vi;
    }
    *vr_out = v[0][0];
    *vi_out = v[0][1];
    *ur_out = v[1][0];
    *ui_out = v[1][1];
}

}  // namespace bc
