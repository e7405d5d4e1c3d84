// Shape derivatives of a DP0 Helmholtz scattering functional (adjoint method).
//
// For A phi = b, u = F phi and a real functional of u, the adjoint vector
// lambda reduces the vertex gradient to three contractions
//   Re(lambda^H dA phi), Re(u^H dF phi), Re(lambda^H db),
// each a sum over element pairs (or elements) of derivatives of quadrature
// sums.  Nothing here forms dA/dx: every pass recomputes the quadrature.
//
// Notation for one element pair (test t, trial s), DP0, one quadrature-point
// pair (x in t, y in s), d = y - x, r = |d|, G = exp(ikr) / (4 pi r),
// z = ikr - 1, c_s = (v1 - v0) x (v2 - v0) of s (so c_s = ie_s n_s),
// u = (d . c_s) / r^2:
//   A_ts = ie_t sum w [ beta G z u + eta ie_s G ]         (DLP + eta SLP)
// with beta = dlp_coeff * normal multiplier of s.  Contracted with
// c' = conj(lambda_t) phi_s ie_t and Gc = c' w G:
//   d/dd    : gd = a1 d + a2 c_s,
//             a1 = [beta u Re(Gc (3 - k^2 r^2 - 3ikr)) + ie_s Re(Gc z eta)] / r^2,
//             a2 = beta Re(Gc z) / r^2
//   d/dc_s  : a2 d
//   d/die_s : Re(Gc eta)
//   d/die_t : Re(Gc (beta z u + eta ie_s)) / ie_t
//   d/dk    : Re(Gc (-beta k r^2 u + (i eta r + eta') ie_s))
// (from dG/dr = G z / r, d(G z / r^2)/dr = G (3 - 3ikr - k^2 r^2) / r^3,
// dG/dk = i r G, d(G z / r^2)/dk = -k G).  x = v0 + xi e1 + eta e2 with
// e1 = v1 - v0, e2 = v2 - v0, so vertex a of t receives -sum N_a(x) gd and
// vertex b of s receives +sum N_b(y) gd; c and ie go through the cross
// product:  d(C . c)/dv1 = e2 x C, d(C . c)/dv2 = C x e1,
// d ie/dv1 = e2 x n, d ie/dv2 = n x e1, and dv0 = -(dv1 + dv2) for both.
//
// The quadrature points are fixed in reference coordinates (regular rule and
// Sauter-Schwab tables alike), so these are exact derivatives of the
// discrete operator; near the singular set every derivative of d is O(r)
// (shared vertices move with both elements), so the singular rules integrate
// the differentiated kernel as they integrate the kernel itself.
#include "common.cuh"
#include "fastmath.cuh"

namespace bc {

// Per-element partial sums, SH_ACC doubles per element (element-major).  For
// the points z of element e (test points when e is the row element, trial
// points when it is the column element) with local coordinates (xi, eta):
//  0-2   sum dF/dz                 (test side -gd, trial side +gd)
//  3-5   sum xi(z) dF/dz
//  6-8   sum eta(z) dF/dz
//  9-11  sum a2 d                  (e as trial: derivative through c_e)
//  12    coefficient of d ie_e     (test: ival / ie_e, trial: ere)
//  13    d/dk
constexpr int SH_ACC = 16;
constexpr int SH_THREADS = 128;
constexpr int SH_TCHUNK = 32;
constexpr int SH_TILES = 8;  // row chunks per block
constexpr int SH_WARPS = SH_THREADS / 32;
constexpr int SHS_WARPS = 4;  // singular kernel: pairs per block (154 registers: 3 blocks per SM)
constexpr int SH_NQ = 6;
constexpr int SH_RED = 13;  // row-element sums reduced across a block

struct ShapeParams {
    const double *g;
    int64_t ne, nv;
    const int32_t *el;
    const int32_t *nm;
    double k, beta, eta_re, eta_im, deta_re, deta_im, ident;
    const double2 *phi, *lam, *u;
    double *acc, *vgrad, *kgrad;
    int64_t npairs;
    const double2 *tp, *sp;
    const double *w;
    const int32_t *te, *se, *toff, *soff, *woff, *npts;
    int ndir;
    int phase_class;
    const double *dirs;
    double ff_beta, ff_eta_re, ff_eta_im, ff_deta_re, ff_deta_im;
    double inc[3];
    double rhs_re, rhs_im;
    double scale_op, scale_ff, scale_rhs;
    void *out;
};

// gd = a1 d / r^2 + a2 c_s is formed by the caller: the symmetric sweep adds
// the two ordered pairs' gradients before multiplying by d.
struct QpeTerms {
    double a1;  // a1 r^2
    double a2, ival, ere, kval;
};

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// One ordered quadrature-point pair of the combined kernel.  (gr, gi) = w
// exp(ik(r - r_c)) / (4 pi r) and (cre, cim) = conj(lambda_t) phi_s ie_t
// exp(ik r_c), so Gc = c' w G; d = y - x runs from the test point to the trial
// point.  bcs = beta c_s (the trial normal vector times beta), so the returned
// a2 lacks its factor beta: callers multiply a2 d sums by beta and use a2 bcs
// for a2 c_s.
__device__ __forceinline__ void qpe_ordered(const double d[3], double r, double rinv2, double gr, double gi,
                                            double cre, double cim, const double bcs[3], double ies,
                                            const ShapeParams &P, QpeTerms &o) {
    const double Gr = cre * gr - cim * gi, Gi = fma(cre, gi, cim * gr);
    const double bu = fma(d[2], bcs[2], fma(d[1], bcs[1], d[0] * bcs[0])) * rinv2;
    const double kr = P.k * r;
    const double Zr = fma(-Gi, kr, -Gr), Zi = fma(Gr, kr, -Gi);  // Gc z
    const double reGcEta = Gr * P.eta_re - Gi * P.eta_im;
    const double reGzEta = Zr * P.eta_re - Zi * P.eta_im;
    const double t1 = fma(Gr, 3.0 - kr * kr, 3.0 * kr * Gi);  // Re(Gc (3 - k^2 r^2 - 3ikr))
    o.a1 = fma(bu, t1, ies * reGzEta);
    o.a2 = Zr * rinv2;
    o.ival = fma(bu, Zr, ies * reGcEta);
    o.ere = reGcEta;
    const double er = P.deta_re - P.eta_im * r, ei = fma(P.eta_re, r, P.deta_im);
    o.kval = fma(-bu * (kr * r), Gr, ies * (Gr * er - Gi * ei));
}

// exp(i theta) for the phase offset theta = k (r - r_c) of class PHC (0: any
// argument, 1: |theta| <= 1, 2: |theta| <= 1/2).
template <int PHC>
__device__ __forceinline__ void phase64(double th, double *s, double *c) {
    if (PHC == 2)
        sincos_half64(th, s, c);
    else if (PHC == 1)
        sincos_small64(th, s, c);
    else
        sincos_cw64(th, s, c);
}

__device__ __forceinline__ bool touches(const int *a, int b0, int b1, int b2) {
    return (a[0] == b0) | (a[0] == b1) | (a[0] == b2) | (a[1] == b0) | (a[1] == b1) | (a[1] == b2) | (a[2] == b0) |
           (a[2] == b1) | (a[2] == b2);
}

struct ShapeTile {
    double x[SH_TCHUNK][SH_NQ][3];
    double cr[SH_TCHUNK][3];  // ie_i n_i
    double ce[SH_TCHUNK][3];  // centroid
    double2 lc[SH_TCHUNK];    // conj(lambda_i) ie_i
    double2 ph[SH_TCHUNK];    // phi_i
    double ie[SH_TCHUNK];
    double bet[SH_TCHUNK];
    int v[SH_TCHUNK][3];
    double red[SH_WARPS][SH_TCHUNK][SH_RED];
};

// Regular pairs, symmetric sweep: one thread per column element j, rows i < j
// staged SH_TCHUNK at a time, SH_TILES chunks per block.  Each unordered pair
// gives the ordered pairs (i, j) (test i, trial j) and (j, i) (test j, trial
// i) from one evaluation of r and the phase.  Column sums stay in registers
// for the whole block; row sums are reduced over the warp (shuffles), then
// over the block's warps (shared memory), then added to the workspace.
template <int PHC>
__global__ void __launch_bounds__(SH_THREADS) shape_regular(ShapeParams P, QuadRule rule) {
    const int64_t row0 = (int64_t)blockIdx.y * SH_TILES * SH_TCHUNK;
    const int64_t col0 = (int64_t)blockIdx.x * SH_THREADS;
    if (row0 >= col0 + SH_THREADS) return;  // the whole block lies below the diagonal
    __shared__ ShapeTile sb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t s = col0 + threadIdx.x;
    const bool active = s < P.ne;
    double y[SH_NQ][3], cs[3] = {0.0, 0.0, 0.0}, sc[3] = {0.0, 0.0, 0.0}, v0s[3] = {0.0, 0.0, 0.0};
    double ies = 0.0, ies_inv = 0.0, bet = 0.0;
    double2 phs = make_double2(0.0, 0.0), ls = make_double2(0.0, 0.0);
    int sv0 = -1, sv1 = -1, sv2 = -1;
    if (active) {
        Geom gs;
        load_geom(P.g, P.ne, s, 1.0, gs);
#pragma unroll
        for (int q = 0; q < SH_NQ; ++q) to_global(gs, rule.x[q], rule.y[q], y[q]);
#pragma unroll
        bet = P.beta * (P.nm ? (double)P.nm[s] : 1.0);
        for (int c = 0; c < 3; ++c) {
            cs[c] = bet * gs.n[c] * gs.ie;
            sc[c] = __ldg(P.g + (22 + c) * P.ne + s);
            v0s[c] = gs.v0[c];
        }
        ies = gs.ie;
        ies_inv = 1.0 / gs.ie;
        phs = P.phi[s];
        const double2 l = P.lam[s];
        ls = make_double2(l.x * gs.ie, -l.y * gs.ie);  // conj(lambda_j) ie_j
        sv0 = P.el[3 * s];
        sv1 = P.el[3 * s + 1];
        sv2 = P.el[3 * s + 2];
    } else {
#pragma unroll
        for (int q = 0; q < SH_NQ; ++q) y[q][0] = y[q][1] = y[q][2] = 0.0;
    }
    // column sums: dF/dy per column quadrature point (fields 0-8 are formed from
    // them at the end), then fields 9-13 of the workspace layout
    double cQ[SH_NQ][3], cC[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < SH_NQ; ++q) cQ[q][0] = cQ[q][1] = cQ[q][2] = 0.0;
    double cI = 0.0, cK = 0.0;

    for (int tile = 0; tile < SH_TILES; ++tile) {
        const int64_t t0 = row0 + (int64_t)tile * SH_TCHUNK;
        if (t0 >= P.ne || t0 >= col0 + SH_THREADS) break;  // uniform over the block
        const int tcount = (int)min((int64_t)SH_TCHUNK, P.ne - t0);
        __syncthreads();  // previous chunk's shared data fully consumed
        for (int idx = threadIdx.x; idx < tcount; idx += SH_THREADS) {
            const int64_t t = t0 + idx;
            Geom g;
            load_geom(P.g, P.ne, t, 1.0, g);
#pragma unroll
            for (int p = 0; p < SH_NQ; ++p) to_global(g, rule.x[p], rule.y[p], sb.x[idx][p]);
            const double bi = P.beta * (P.nm ? (double)P.nm[t] : 1.0);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                sb.cr[idx][c] = bi * g.n[c] * g.ie;
                sb.ce[idx][c] = __ldg(P.g + (22 + c) * P.ne + t);
                sb.v[idx][c] = P.el[3 * t + c];
            }
            const double2 l = P.lam[t];
            sb.lc[idx] = make_double2(l.x * g.ie, -l.y * g.ie);
            sb.ph[idx] = P.phi[t];
            sb.ie[idx] = g.ie;
            sb.bet[idx] = bi;
        }
        __syncthreads();
        for (int tt = 0; tt < tcount; ++tt) {
            const int64_t row = t0 + tt;
            double rs[SH_RED];  // row sums of this pair
#pragma unroll
            for (int f = 0; f < SH_RED; ++f) rs[f] = 0.0;
            const bool skip = !active || row >= s || touches(sb.v[tt], sv0, sv1, sv2);
            if (!skip) {
                // pair phase exp(i k r_c) folded into both contraction coefficients
                const double D0 = sc[0] - sb.ce[tt][0], D1 = sc[1] - sb.ce[tt][1], D2 = sc[2] - sb.ce[tt][2];
                const double rc = sqrt(fma(D2, D2, fma(D1, D1, D0 * D0)));
                double pcs = 1.0, psn = 0.0;
                const double krc = P.k * rc;
                if (PHC > 0) sincos_cw64(krc, &psn, &pcs);
                const double2 lt = sb.lc[tt], pt = sb.ph[tt];
                // ordered (i, j): conj(lambda_i) ie_i phi_j;  (j, i): conj(lambda_j) ie_j phi_i
                double c1r = lt.x * phs.x - lt.y * phs.y, c1i = fma(lt.x, phs.y, lt.y * phs.x);
                double c2r = ls.x * pt.x - ls.y * pt.y, c2i = fma(ls.x, pt.y, ls.y * pt.x);
                if (PHC > 0) {
                    const double a = c1r * pcs - c1i * psn, b = fma(c1r, psn, c1i * pcs);
                    c1r = a;
                    c1i = b;
                    const double e = c2r * pcs - c2i * psn, f = fma(c2r, psn, c2i * pcs);
                    c2r = e;
                    c2i = f;
                }
                const double iet = sb.ie[tt], iet_inv = 1.0 / iet;
                const double ct[3] = {sb.cr[tt][0], sb.cr[tt][1], sb.cr[tt][2]};
                // sums over the pair's points of G and r G (the eta and d eta / dk terms are linear in G
                // with per-pair coefficients) and of the u-weighted terms of the area and k derivatives
                double sgr = 0.0, sgi = 0.0, srgr = 0.0, srgi = 0.0, iz1 = 0.0, iz2 = 0.0, kz = 0.0;
                for (int p = 0; p < SH_NQ; ++p) {
                    const double x0 = sb.x[tt][p][0], x1 = sb.x[tt][p][1], x2 = sb.x[tt][p][2];
                    const double wp = rule.w[p] * BC_INV_4PI;
                    // (y - x).(beta_j c_j) = (v0_j - x).(beta_j c_j): y lies in the plane of j
                    const double xs = fma(v0s[2] - x2, cs[2], fma(v0s[1] - x1, cs[1], (v0s[0] - x0) * cs[0]));
                    double pp[3] = {0.0, 0.0, 0.0};  // row-element point derivative at x_p
#pragma unroll
                    for (int q = 0; q < SH_NQ; ++q) {
                        const double d[3] = {y[q][0] - x0, y[q][1] - x1, y[q][2] - x2};
                        const double r2 = fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0]));
                        const double rinv = rsqrt64(r2);
                        const double r = r2 * rinv;
                        const double rinv2 = rinv * rinv;
                        double sn, cn;
                        if (PHC > 0)
                            phase64<PHC>(fma(P.k, r, -krc), &sn, &cn);
                        else
                            sincos_cw64(P.k * r, &sn, &cn);
                        const double f = (wp * rule.w[q]) * rinv;
                        const double gr = cn * f, gi = sn * f;
                        sgr += gr;
                        sgi += gi;
                        srgr = fma(r, gr, srgr);
                        srgi = fma(r, gi, srgi);
                        const double kq = P.k * r;
                        const double t13 = fma(-kq, kq, 3.0), k3 = 3.0 * kq;
                        // (i, j): x in i (test), y in j (trial), d = y - x, Gc = c1 G, z = ikr - 1
                        const double G1r = c1r * gr - c1i * gi, G1i = fma(c1r, gi, c1i * gr);
                        const double Z1r = fma(-G1i, kq, -G1r), Z1i = fma(G1r, kq, -G1i);
                        const double bu1 = xs * rinv2;
                        const double a1_1 = fma(bu1, fma(G1r, t13, k3 * G1i), ies * (Z1r * P.eta_re - Z1i * P.eta_im));
                        const double a2_1 = Z1r * rinv2;
                        // (j, i): test point y, trial point x, d' = -d, Gc = c2 G
                        const double G2r = c2r * gr - c2i * gi, G2i = fma(c2r, gi, c2i * gr);
                        const double Z2r = fma(-G2i, kq, -G2r), Z2i = fma(G2r, kq, -G2i);
                        const double bu2 = -fma(d[2], ct[2], fma(d[1], ct[1], d[0] * ct[0])) * rinv2;
                        const double a1_2 = fma(bu2, fma(G2r, t13, k3 * G2i), iet * (Z2r * P.eta_re - Z2i * P.eta_im));
                        const double a2_2 = Z2r * rinv2;
                        iz1 = fma(bu1, Z1r, iz1);
                        iz2 = fma(bu2, Z2r, iz2);
                        kz = fma(fma(bu1, G1r, bu2 * G2r), kq * r, kz);
                        // column element j: trial of (i, j) (+gd1), test of (j, i) (-gd2)
                        // gd of (i, j) minus gd of (j, i): (a1_1 + a1_2) d / r^2 + a2_1 c_j - a2_2 c_i
                        const double a1s = (a1_1 + a1_2) * rinv2;
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const double gj = fma(a1s, d[c], fma(a2_1, cs[c], -a2_2 * ct[c]));
                            cQ[q][c] += gj;
                            cC[c] = fma(a2_1, d[c], cC[c]);
                            pp[c] -= gj;  // row element i: test of (i, j) (-gd1), trial of (j, i) (+gd2)
                            rs[9 + c] = fma(-a2_2, d[c], rs[9 + c]);
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        rs[c] += pp[c];
                        rs[3 + c] = fma(rule.x[p], pp[c], rs[3 + c]);
                        rs[6 + c] = fma(rule.y[p], pp[c], rs[6 + c]);
                    }
                }
                // ere_o = Re(eta c_o G) and ival_o = bu_o Re(c_o G z) + ie_o ere_o summed over the points:
                // E_o = Re(eta c_o sum G); d/dk: Re(c_o (d eta + i r eta) G) = Re(dc_o sum G) - Im(ec_o sum r G)
                const double ec1r = P.eta_re * c1r - P.eta_im * c1i, ec1i = fma(P.eta_re, c1i, P.eta_im * c1r);
                const double ec2r = P.eta_re * c2r - P.eta_im * c2i, ec2i = fma(P.eta_re, c2i, P.eta_im * c2r);
                const double dc1r = P.deta_re * c1r - P.deta_im * c1i, dc1i = fma(P.deta_re, c1i, P.deta_im * c1r);
                const double dc2r = P.deta_re * c2r - P.deta_im * c2i, dc2i = fma(P.deta_re, c2i, P.deta_im * c2r);
                const double e1 = ec1r * sgr - ec1i * sgi, e2 = ec2r * sgr - ec2i * sgi;
                const double k1 = (dc1r * sgr - dc1i * sgi) - fma(ec1r, srgi, ec1i * srgr);
                const double k2 = (dc2r * sgr - dc2i * sgi) - fma(ec2r, srgi, ec2i * srgr);
                cI += fma(ies_inv, fma(iet, e2, iz2), e1);
                rs[12] += fma(iet_inv, fma(ies, e1, iz1), e2);
                cK += fma(ies, k1, fma(iet, k2, -kz));
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) rs[9 + c] *= sb.bet[tt];  // a2 d sums lack beta_i
#pragma unroll
            for (int f = 0; f < SH_RED; ++f) rs[f] = warp_sum(rs[f]);
            if (lane == 0)
#pragma unroll
                for (int f = 0; f < SH_RED; ++f) sb.red[warp][tt][f] = rs[f];
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < tcount * SH_RED; idx += SH_THREADS) {
            const int tt = idx / SH_RED, f = idx - SH_RED * (idx / SH_RED);
            double v = 0.0;
#pragma unroll
            for (int wi = 0; wi < SH_WARPS; ++wi) v += sb.red[wi][tt][f];
            if (v != 0.0) atomicAdd(P.acc + (t0 + tt) * SH_ACC + f, v);
        }
    }
    if (active) {
        double *a = P.acc + s * SH_ACC;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double cT = 0.0, cX = 0.0, cY = 0.0;
#pragma unroll
            for (int q = 0; q < SH_NQ; ++q) {
                cT += cQ[q][c];
                cX = fma(rule.x[q], cQ[q][c], cX);
                cY = fma(rule.y[q], cQ[q][c], cY);
            }
            atomicAdd(a + c, cT);
            atomicAdd(a + 3 + c, cX);
            atomicAdd(a + 6 + c, cY);
            atomicAdd(a + 9 + c, bet * cC[c]);  // a2 d sums lack beta_j
        }
        atomicAdd(a + 12, cI);
        atomicAdd(a + 13, cK);
    }
}

// Singular pairs: one warp per ordered pair, lanes over its Sauter-Schwab points.
__global__ void __launch_bounds__(32 * SHS_WARPS) shape_singular(ShapeParams P) {
    const int lane = threadIdx.x & 31;
    const int64_t k = (int64_t)blockIdx.x * SHS_WARPS + (threadIdx.x >> 5);
    if (k >= P.npairs) return;
    const int64_t t = P.te[k], s = P.se[k];
    Geom gt, gs;
    load_geom(P.g, P.ne, t, 1.0, gt);
    load_geom(P.g, P.ne, s, 1.0, gs);
    const double2 l = P.lam[t], ph = P.phi[s];
    const double cre = (l.x * ph.x + l.y * ph.y) * gt.ie, cim = (l.x * ph.y - l.y * ph.x) * gt.ie;
    const double bet = P.beta * (P.nm ? (double)P.nm[s] : 1.0);
    const double cs[3] = {bet * gs.n[0] * gs.ie, bet * gs.n[1] * gs.ie, bet * gs.n[2] * gs.ie};
    const double ies = gs.ie;
    // 0-2 sum gd, 3-5 xi(x) gd, 6-8 eta(x) gd, 9-11 xi(y) gd, 12-14 eta(y) gd, 15-17 a2 d, 18 ival, 19 ere, 20 k
    double a[21];
#pragma unroll
    for (int f = 0; f < 21; ++f) a[f] = 0.0;
    const int64_t toff = P.toff[k], soff = P.soff[k], woff = P.woff[k];
    const int n = P.npts[k];
    for (int m = lane; m < n; m += 32) {
        const double2 tpm = P.tp[toff + m], spm = P.sp[soff + m];
        const double w = P.w[woff + m];
        double x[3], y[3];
        to_global(gt, tpm.x, tpm.y, x);
        to_global(gs, spm.x, spm.y, y);
        const double d[3] = {y[0] - x[0], y[1] - x[1], y[2] - x[2]};
        const double r2 = fma(d[2], d[2], fma(d[1], d[1], d[0] * d[0]));
        const double rinv = rsqrt64(r2);
        const double r = r2 * rinv;
        double sn, cn;
        sincos_cw64(P.k * r, &sn, &cn);
        const double f = w * rinv * BC_INV_4PI;
        QpeTerms o;
        const double rinv2 = rinv * rinv;
        qpe_ordered(d, r, rinv2, cn * f, sn * f, cre, cim, cs, ies, P, o);
        const double a1 = o.a1 * rinv2;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double gd = fma(a1, d[c], o.a2 * cs[c]);
            a[c] += gd;
            a[3 + c] = fma(tpm.x, gd, a[3 + c]);
            a[6 + c] = fma(tpm.y, gd, a[6 + c]);
            a[9 + c] = fma(spm.x, gd, a[9 + c]);
            a[12 + c] = fma(spm.y, gd, a[12 + c]);
            a[15 + c] = fma(o.a2, d[c], a[15 + c]);
        }
        a[18] += o.ival;
        a[19] += o.ere;
        a[20] += o.kval;
    }
#pragma unroll
    for (int f = 0; f < 21; ++f) a[f] = warp_sum(a[f]);
    if (lane != 0) return;
    double *at = P.acc + t * SH_ACC, *as = P.acc + s * SH_ACC;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        atomicAdd(at + c, -a[c]);
        atomicAdd(at + 3 + c, -a[3 + c]);
        atomicAdd(at + 6 + c, -a[6 + c]);
        atomicAdd(as + c, a[c]);
        atomicAdd(as + 3 + c, a[9 + c]);
        atomicAdd(as + 6 + c, a[12 + c]);
        atomicAdd(as + 9 + c, bet * a[15 + c]);
    }
    atomicAdd(at + 12, a[18] / gt.ie);
    atomicAdd(as + 12, a[19]);
    atomicAdd(as + 13, a[20]);
}

// Vertex gradient of one element from "trial-type" sums: sum of a gradient
// with respect to points y (T, sum xi(y) ., sum eta(y) .), a vector C
// contracted with c = e1 x e2, and a coefficient of ie.
__device__ __forceinline__ void trial_chain(const Geom &g, const double di[3][3], const double T[3],
                                            const double X[3], const double Y[3], const double C[3], double cie,
                                            double gv[3][3]) {
    double w1[3], w2[3];
    cross3(g.j1, C, w1);
    cross3(C, g.j0, w2);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        gv[0][c] += T[c] - X[c] - Y[c] - w1[c] - w2[c] + cie * di[0][c];
        gv[1][c] += X[c] + w1[c] + cie * di[1][c];
        gv[2][c] += Y[c] + w2[c] + cie * di[2][c];
    }
}

// One thread per element: chain rule of the operator sums, the far-field and
// right-hand-side terms, scatter to the vertices, and the wavenumber sum.
__global__ void __launch_bounds__(128) shape_finish(ShapeParams P, QuadRule rule) {
    __shared__ double s_k[4];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double kloc = 0.0;
    if (e < P.ne) {
        Geom g;
        load_geom(P.g, P.ne, e, 1.0, g);
        const double nmv = P.nm ? (double)P.nm[e] : 1.0;
        double di[3][3];
        cross3(g.j1, g.n, di[1]);
        cross3(g.n, g.j0, di[2]);
#pragma unroll
        for (int c = 0; c < 3; ++c) di[0][c] = -(di[1][c] + di[2][c]);
        double gv[3][3];
#pragma unroll
        for (int v = 0; v < 3; ++v) gv[v][0] = gv[v][1] = gv[v][2] = 0.0;

        if (P.scale_op != 0.0) {
            const double *a = P.acc + e * SH_ACC;
            const double2 l = P.lam[e], ph = P.phi[e];
            double go[3][3];
#pragma unroll
            for (int v = 0; v < 3; ++v) go[v][0] = go[v][1] = go[v][2] = 0.0;
            const double idc = (l.x * ph.x + l.y * ph.y) * P.ident * 0.5;  // identity: A_ee += ident ie_e / 2
            trial_chain(g, di, a, a + 3, a + 6, a + 9, a[12] + idc, go);
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int c = 0; c < 3; ++c) gv[v][c] = P.scale_op * go[v][c];
            kloc = P.scale_op * a[13];
        }

        if (P.scale_ff != 0.0 && P.ndir > 0) {
            // F_je = sum_q w_q / (4 pi) B_j exp(-i k d_j . y_q), B_j = -i k beta (d_j . c) + eta ie
            const double2 ph = P.phi[e];
            const double bet = P.ff_beta * nmv;
            double c_e[3];
            cross3(g.j0, g.j1, c_e);
            double yq[SH_NQ][3];
#pragma unroll
            for (int q = 0; q < SH_NQ; ++q) to_global(g, rule.x[q], rule.y[q], yq[q]);
            double T[3] = {0.0, 0.0, 0.0}, X[3] = {0.0, 0.0, 0.0}, Y[3] = {0.0, 0.0, 0.0}, C[3] = {0.0, 0.0, 0.0};
            double cie = 0.0, kf = 0.0;
            for (int j = 0; j < P.ndir; ++j) {
                const double dj[3] = {P.dirs[3 * j], P.dirs[3 * j + 1], P.dirs[3 * j + 2]};
                const double2 uj = P.u[j];
                // cj = conj(u_j) phi_e
                const double cjr = uj.x * ph.x + uj.y * ph.y, cji = uj.x * ph.y - uj.y * ph.x;
                const double dc = dj[0] * c_e[0] + dj[1] * c_e[1] + dj[2] * c_e[2];
                const double Br = P.ff_eta_re * g.ie, Bi = fma(-P.k * bet, dc, P.ff_eta_im * g.ie);
                for (int q = 0; q < rule.nq; ++q) {
                    const double dy = dj[0] * yq[q][0] + dj[1] * yq[q][1] + dj[2] * yq[q][2];
                    double sn, cn;
                    sincos_cw64(P.k * dy, &sn, &cn);  // exp(-i k d.y) = (cn, -sn)
                    const double f = rule.w[q] * BC_INV_4PI;
                    const double Vr = (cjr * cn + cji * sn) * f, Vi = (cji * cn - cjr * sn) * f;
                    const double VBi = fma(Vr, Bi, Vi * Br);  // Im(V B)
                    const double gy = P.k * VBi;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const double gyc = gy * dj[c];
                        T[c] += gyc;
                        X[c] = fma(rule.x[q], gyc, X[c]);
                        Y[c] = fma(rule.y[q], gyc, Y[c]);
                        C[c] = fma(P.k * bet * Vi, dj[c], C[c]);
                    }
                    cie += Vr * P.ff_eta_re - Vi * P.ff_eta_im;
                    kf += Vr * P.ff_deta_re * g.ie - Vi * fma(-bet, dc, P.ff_deta_im * g.ie) + dy * VBi;
                }
            }
            double gf[3][3];
#pragma unroll
            for (int v = 0; v < 3; ++v) gf[v][0] = gf[v][1] = gf[v][2] = 0.0;
            trial_chain(g, di, T, X, Y, C, cie, gf);
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int c = 0; c < 3; ++c) gv[v][c] = fma(P.scale_ff, gf[v][c], gv[v][c]);
            kloc = fma(P.scale_ff, kf, kloc);
        }

        if (P.scale_rhs != 0.0) {
            // b_e = rho ie sum_p w_p exp(i k d_inc . x_p), contracted with conj(lambda_e)
            const double2 l = P.lam[e];
            const double cbr = l.x * P.rhs_re + l.y * P.rhs_im, cbi = l.x * P.rhs_im - l.y * P.rhs_re;
            double gb[3][3];
#pragma unroll
            for (int v = 0; v < 3; ++v) gb[v][0] = gb[v][1] = gb[v][2] = 0.0;
            double cie = 0.0, kb = 0.0;
            for (int p = 0; p < rule.nq; ++p) {
                double x[3];
                to_global(g, rule.x[p], rule.y[p], x);
                const double dx = P.inc[0] * x[0] + P.inc[1] * x[1] + P.inc[2] * x[2];
                double sn, cn;
                sincos_cw64(P.k * dx, &sn, &cn);
                const double Er = (cbr * cn - cbi * sn) * rule.w[p], Ei = fma(cbr, sn, cbi * cn) * rule.w[p];
                cie += Er;
                const double gx = -P.k * Ei * g.ie;
                const double nb[3] = {1.0 - rule.x[p] - rule.y[p], rule.x[p], rule.y[p]};
#pragma unroll
                for (int v = 0; v < 3; ++v)
#pragma unroll
                    for (int c = 0; c < 3; ++c) gb[v][c] = fma(nb[v] * gx, P.inc[c], gb[v][c]);
                kb -= dx * Ei * g.ie;
            }
#pragma unroll
            for (int v = 0; v < 3; ++v)
#pragma unroll
                for (int c = 0; c < 3; ++c) gv[v][c] = fma(P.scale_rhs, fma(cie, di[v][c], gb[v][c]), gv[v][c]);
            kloc = fma(P.scale_rhs, kb, kloc);
        }

#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const int64_t vid = P.el[3 * e + v];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (gv[v][c] != 0.0) atomicAdd(P.vgrad + 3 * vid + c, gv[v][c]);
        }
    }
    kloc = warp_sum(kloc);
    if ((threadIdx.x & 31) == 0) s_k[threadIdx.x >> 5] = kloc;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double v = s_k[0] + s_k[1] + s_k[2] + s_k[3];
        if (v != 0.0) atomicAdd(P.kgrad, v);
    }
}

// F[j, e]: thread per entry, elements fastest (coalesced stores).
__global__ void __launch_bounds__(128) shape_farfield(ShapeParams P, QuadRule rule) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.ne * (int64_t)P.ndir) return;
    const int64_t j = idx / P.ne, e = idx - j * P.ne;
    Geom g;
    load_geom(P.g, P.ne, e, 1.0, g);
    const double bet = P.ff_beta * (P.nm ? (double)P.nm[e] : 1.0);
    double c_e[3];
    cross3(g.j0, g.j1, c_e);
    const double dj[3] = {P.dirs[3 * j], P.dirs[3 * j + 1], P.dirs[3 * j + 2]};
    const double dc = dj[0] * c_e[0] + dj[1] * c_e[1] + dj[2] * c_e[2];
    const double Br = P.ff_eta_re * g.ie, Bi = fma(-P.k * bet, dc, P.ff_eta_im * g.ie);
    double sr = 0.0, si = 0.0;
    for (int q = 0; q < rule.nq; ++q) {
        double y[3];
        to_global(g, rule.x[q], rule.y[q], y);
        double sn, cn;
        sincos_cw64(P.k * (dj[0] * y[0] + dj[1] * y[1] + dj[2] * y[2]), &sn, &cn);
        sr = fma(rule.w[q], cn, sr);
        si = fma(-rule.w[q], sn, si);
    }
    sr *= BC_INV_4PI;
    si *= BC_INV_4PI;
    reinterpret_cast<double2 *>(P.out)[idx] = make_double2(sr * Br - si * Bi, fma(sr, Bi, si * Br));
}

__global__ void __launch_bounds__(128) shape_plane_wave(ShapeParams P, QuadRule rule) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.ne) return;
    Geom g;
    load_geom(P.g, P.ne, e, 1.0, g);
    double sr = 0.0, si = 0.0;
    for (int p = 0; p < rule.nq; ++p) {
        double x[3];
        to_global(g, rule.x[p], rule.y[p], x);
        double sn, cn;
        sincos_cw64(P.k * (P.inc[0] * x[0] + P.inc[1] * x[1] + P.inc[2] * x[2]), &sn, &cn);
        sr = fma(rule.w[p], cn, sr);
        si = fma(rule.w[p], sn, si);
    }
    sr *= g.ie;
    si *= g.ie;
    reinterpret_cast<double2 *>(P.out)[e] = make_double2(P.rhs_re * sr - P.rhs_im * si, fma(P.rhs_re, si, P.rhs_im * sr));
}

}  // namespace bc

using namespace bc;

static bool finite_value(double v) { return v == v && v < 1e300 && v > -1e300; }

static int shape_setup(const bemppcuda_shape_args *a, ShapeParams &P, QuadRule &rule, const char *what) {
    if (!a) {
        bc_set_error("%s: null argument struct", what);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->grid.nelements <= 0 || a->grid.nvertices <= 0 || !a->grid.geom || !a->grid.elements) {
        bc_set_error("%s: grid geometry, elements and sizes are required", what);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->nq != SH_NQ || !a->quad_points || !a->quad_weights) {
        bc_set_error("%s: the 6-point regular rule (order 4) is required (got nq = %d)", what, a->nq);
        return BEMPPCUDA_ERR_INVALID;
    }
    const double vals[] = {a->k, a->dlp_coeff, a->eta[0], a->eta[1], a->deta_dk[0], a->deta_dk[1], a->identity,
                           a->ff_dlp_coeff, a->ff_eta[0], a->ff_eta[1], a->ff_deta_dk[0], a->ff_deta_dk[1],
                           a->incident[0], a->incident[1], a->incident[2], a->rhs_coeff[0], a->rhs_coeff[1],
                           a->scale_operator, a->scale_farfield, a->scale_rhs};
    for (double v : vals)
        if (!finite_value(v)) {
            bc_set_error("%s: wavenumber, coefficients and scales must be finite", what);
            return BEMPPCUDA_ERR_INVALID;
        }
    P.g = a->grid.geom;
    P.ne = a->grid.nelements;
    P.nv = a->grid.nvertices;
    P.el = a->grid.elements;
    P.nm = a->normal_mult;
    P.k = a->k;
    P.beta = a->dlp_coeff;
    P.eta_re = a->eta[0];
    P.eta_im = a->eta[1];
    P.deta_re = a->deta_dk[0];
    P.deta_im = a->deta_dk[1];
    P.ident = a->identity;
    P.phi = reinterpret_cast<const double2 *>(a->phi);
    P.lam = reinterpret_cast<const double2 *>(a->lambda);
    P.u = reinterpret_cast<const double2 *>(a->u);
    P.acc = reinterpret_cast<double *>(a->workspace);
    P.vgrad = a->vertex_grad;
    P.kgrad = a->k_grad;
    P.npairs = a->npairs;
    P.tp = reinterpret_cast<const double2 *>(a->test_points);
    P.sp = reinterpret_cast<const double2 *>(a->trial_points);
    P.w = a->weights;
    P.te = a->test_elements;
    P.se = a->trial_elements;
    P.toff = a->test_offsets;
    P.soff = a->trial_offsets;
    P.woff = a->weights_offsets;
    P.npts = a->npoints;
    P.ndir = a->ndirections;
    {
        // |k| (R_i + R_j) bounds the phase offset k (r - r_c) of every regular pair
        const double theta = fabs(a->k) * a->phase_radius;
        P.phase_class = a->phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
    }
    P.dirs = a->directions;
    P.ff_beta = a->ff_dlp_coeff;
    P.ff_eta_re = a->ff_eta[0];
    P.ff_eta_im = a->ff_eta[1];
    P.ff_deta_re = a->ff_deta_dk[0];
    P.ff_deta_im = a->ff_deta_dk[1];
    for (int c = 0; c < 3; ++c) P.inc[c] = a->incident[c];
    P.rhs_re = a->rhs_coeff[0];
    P.rhs_im = a->rhs_coeff[1];
    P.scale_op = a->scale_operator;
    P.scale_ff = a->scale_farfield;
    P.scale_rhs = a->scale_rhs;
    P.out = a->out;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);
    return BEMPPCUDA_OK;
}

extern "C" {

int64_t bemppcuda_shape_workspace_bytes(int64_t nelements) {
    return nelements > 0 ? nelements * SH_ACC * (int64_t)sizeof(double) : 0;
}

int bemppcuda_farfield_matrix_dp0(const bemppcuda_shape_args *a, void *stream) {
    ShapeParams P;
    QuadRule rule;
    int rc = shape_setup(a, P, rule, "farfield_matrix_dp0");
    if (rc) return rc;
    if (P.ndir <= 0 || !P.dirs || !P.out) {
        bc_set_error("farfield_matrix_dp0: directions and an output of ndirections x nelements are required");
        return BEMPPCUDA_ERR_INVALID;
    }
    const int64_t n = P.ne * (int64_t)P.ndir;
    shape_farfield<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(P, rule);
    return bc_check_launch("farfield_matrix_dp0");
}

int bemppcuda_plane_wave_dp0(const bemppcuda_shape_args *a, void *stream) {
    ShapeParams P;
    QuadRule rule;
    int rc = shape_setup(a, P, rule, "plane_wave_dp0");
    if (rc) return rc;
    if (!P.out) {
        bc_set_error("plane_wave_dp0: output vector required");
        return BEMPPCUDA_ERR_INVALID;
    }
    shape_plane_wave<<<(unsigned)((P.ne + 127) / 128), 128, 0, (cudaStream_t)stream>>>(P, rule);
    return bc_check_launch("plane_wave_dp0");
}

int bemppcuda_shape_adjoint_dp0(const bemppcuda_shape_args *a, void *stream) {
    ShapeParams P;
    QuadRule rule;
    int rc = shape_setup(a, P, rule, "shape_adjoint_dp0");
    if (rc) return rc;
    if (!P.vgrad || !P.kgrad) {
        bc_set_error("shape_adjoint_dp0: vertex_grad and k_grad outputs are required");
        return BEMPPCUDA_ERR_INVALID;
    }
    const bool op = P.scale_op != 0.0, ff = P.scale_ff != 0.0, rhs = P.scale_rhs != 0.0;
    if ((op && (!P.phi || !P.lam)) || (ff && (!P.phi || !P.u || !P.dirs || P.ndir <= 0)) || (rhs && !P.lam)) {
        bc_set_error("shape_adjoint_dp0: phi / lambda / u / directions missing for a term with a nonzero scale");
        return BEMPPCUDA_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (op) {
        const int64_t need = bemppcuda_shape_workspace_bytes(P.ne);
        if (!P.acc || a->workspace_bytes < need) {
            bc_set_error("shape_adjoint_dp0: workspace of %lld bytes required (got %lld)", (long long)need,
                         (long long)a->workspace_bytes);
            return BEMPPCUDA_ERR_WORKSPACE;
        }
        if (P.npairs < 0 || (P.npairs > 0 && (!P.tp || !P.sp || !P.w || !P.te || !P.se || !P.toff || !P.soff ||
                                              !P.woff || !P.npts))) {
            bc_set_error("shape_adjoint_dp0: singular pair tables missing");
            return BEMPPCUDA_ERR_INVALID;
        }
        if (cudaMemsetAsync(P.acc, 0, need, st) != cudaSuccess) return bc_check_launch("shape_adjoint_dp0 memset");
        const int64_t by = (P.ne + SH_TCHUNK * SH_TILES - 1) / (SH_TCHUNK * SH_TILES);
        if (by > 65535) {
            bc_set_error("shape_adjoint_dp0: %lld elements exceed the launch grid", (long long)P.ne);
            return BEMPPCUDA_ERR_UNSUPPORTED;
        }
        dim3 grid((unsigned)((P.ne + SH_THREADS - 1) / SH_THREADS), (unsigned)by);
        if (P.phase_class == 2)
            shape_regular<2><<<grid, SH_THREADS, 0, st>>>(P, rule);
        else if (P.phase_class == 1)
            shape_regular<1><<<grid, SH_THREADS, 0, st>>>(P, rule);
        else
            shape_regular<0><<<grid, SH_THREADS, 0, st>>>(P, rule);
        rc = bc_check_launch("shape_adjoint_dp0 regular pairs");
        if (rc) return rc;
        if (P.npairs > 0) {
            shape_singular<<<(unsigned)((P.npairs + SHS_WARPS - 1) / SHS_WARPS), 32 * SHS_WARPS, 0, st>>>(P);
            rc = bc_check_launch("shape_adjoint_dp0 singular pairs");
            if (rc) return rc;
        }
    }
    shape_finish<<<(unsigned)((P.ne + 127) / 128), 128, 0, st>>>(P, rule);
    return bc_check_launch("shape_adjoint_dp0 element pass");
}

}  // extern "C"
