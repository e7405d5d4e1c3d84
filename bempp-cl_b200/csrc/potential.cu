// Potential and far-field evaluation: u(x) = sum over support elements and
// quadrature points of G(x, y_eq) c_eq.
//
// Replaces default_scalar_potential_kernel (numba_kernels.py:1788-1849),
// maxwell_efield_potential (:2281-2359), maxwell_mfield_potential
// (:2363-2433), maxwell_efield_far_field (:2437-2503) and
// maxwell_mfield_far_field (:2507-2570).
//
// Two launches on one stream:
//  1. potential_sources: one thread per (element, quadrature point) writes the
//     source point, normal and weighted coefficient(s) field-major into the
//     caller's workspace (the reference's `tmp` arrays).
//  2. potential_scalar (Laplace, Helmholtz and modified Helmholtz single /
//     double layer): a thread per evaluation point walks the sources staged
//     in shared memory; see the comment above the kernel.
//     potential_eval (far fields, Maxwell): one warp owns PPW evaluation points;
//     its lanes stride over the sources with coalesced loads, accumulate per
//     point in FP64 and combine with xor-shuffle reductions; lane 0 writes.
#include <algorithm>

#include "dp0.cuh"  // common.cuh, and the packed FP32 helpers of the mixed kernels

namespace bc {

// workspace fields per source: y(3) n(3) then
//   scalar:  cre cim, and fields 8-10 at index ei (< nsupport) hold element ei's centroid
//   Maxwell: c0re c0im c1re c1im c2re c2im dre dim
constexpr int SRC_FIELDS = 14;
constexpr int POT_PPW = 4;
constexpr int POT_WARPS = 4;

struct PotParams {
    const double *g;
    int64_t ne;
    const uint32_t *support;
    int64_t nsupport;
    const int32_t *nm;
    int nshape;
    int nq;
    const double *coeff;  // complex (ne * nshape)
    double *src;          // workspace SRC_FIELDS * nsrc
    int64_t nsrc;
    const double *points;  // (npoints, 3)
    int64_t npoints;
    double *result;  // complex (kdim, npoints)
    double p[4];
};

template <bool MAXWELL>
__global__ void potential_sources(PotParams prm, QuadRule rule) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= prm.nsrc) return;
    const int64_t ei = k / prm.nq;
    const int q = (int)(k - ei * prm.nq);
    const int64_t e = prm.support[ei];
    Geom g;
    load_geom(prm.g, prm.ne, e, prm.nm ? (double)prm.nm[e] : 1.0, g);
    double y[3];
    to_global(g, rule.x[q], rule.y[q], y);
    double *o = prm.src;
    const int64_t n = prm.nsrc;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        o[d * n + k] = y[d];
        o[(3 + d) * n + k] = g.n[d];
    }
    const double2 *x = reinterpret_cast<const double2 *>(prm.coeff) + e * prm.nshape;
    if (!MAXWELL) {
        double phi[3];
        scalar_shape(prm.nshape, rule.x[q], rule.y[q], phi);
        double cr = 0.0, ci = 0.0;
        for (int i = 0; i < prm.nshape; ++i) {
            const double2 xi = x[i];
            const double f = g.ie * rule.w[q] * phi[i];
            cr = fma(f, xi.x, cr);
            ci = fma(f, xi.y, ci);
        }
        o[6 * n + k] = cr;
        o[7 * n + k] = ci;
        if (q == 0) {
            // element centroid, indexed by support position, for the phase factoring of potential_scalar
            double c[3];
            to_global(g, 1.0 / 3.0, 1.0 / 3.0, c);
#pragma unroll
            for (int d = 0; d < 3; ++d) o[(8 + d) * n + ei] = c[d];
        }
    } else {
        double b[3][3];
        rwg_values(g, rule.x[q], rule.y[q], b);
        double vr[3] = {0, 0, 0}, vi[3] = {0, 0, 0}, dr = 0.0, di = 0.0;
        for (int i = 0; i < 3; ++i) {
            const double2 xi = x[i];
            const double el = edge_length(prm.g, prm.ne, e, i);
            const double fr = rule.w[q] * xi.x * el, fi = rule.w[q] * xi.y * el;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                vr[d] += fr * b[i][d] * g.ie;
                vi[d] += fi * b[i][d] * g.ie;
            }
            dr += 2.0 * fr;
            di += 2.0 * fi;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            o[(6 + 2 * d) * n + k] = vr[d];
            o[(7 + 2 * d) * n + k] = vi[d];
        }
        o[12 * n + k] = dr;
        o[13 * n + k] = di;
    }
}

template <int ASM, int K>
__global__ void __launch_bounds__(32 * POT_WARPS) potential_eval(PotParams prm) {
    constexpr bool FAR = (K == BEMPPCUDA_FARFIELD_SLP || K == BEMPPCUDA_FARFIELD_DLP);
    constexpr int KD = (ASM == BEMPPCUDA_ASM_SCALAR) ? 1 : 3;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * POT_WARPS + (threadIdx.x >> 5);
    const int64_t p0 = warp * POT_PPW;
    if (p0 >= prm.npoints) return;
    double xp[POT_PPW][3];
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j) {
        const int64_t pj = min(p0 + j, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) xp[j][d] = prm.points[3 * pj + d];
    }
    double ar[POT_PPW][KD], ai[POT_PPW][KD];
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j)
#pragma unroll
        for (int d = 0; d < KD; ++d) ar[j][d] = ai[j][d] = 0.0;
    const double kr = prm.p[0], ki = prm.p[1];
    const double zero[3] = {0.0, 0.0, 0.0};
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t k = lane; k < n; k += 32) {
        const double y[3] = {o[k], o[n + k], o[2 * n + k]};
        const double ny[3] = {o[3 * n + k], o[4 * n + k], o[5 * n + k]};
        if (ASM == BEMPPCUDA_ASM_SCALAR) {
            const double cr = o[6 * n + k], ci = o[7 * n + k];
#pragma unroll
            for (int j = 0; j < POT_PPW; ++j) {
                const cplx kv = greens<K>(xp[j], y, zero, ny, prm.p);
                ar[j][0] += kv.re * cr - kv.im * ci;
                ai[j][0] += kv.re * ci + kv.im * cr;
            }
        } else {
            cplx v[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) v[d] = {o[(6 + 2 * d) * n + k], o[(7 + 2 * d) * n + k]};
            const cplx dv = {o[12 * n + k], o[13 * n + k]};
            const cplx ik = {-ki, kr};
#pragma unroll
            for (int j = 0; j < POT_PPW; ++j) {
                const cplx kv = greens<K>(xp[j], y, zero, ny, prm.p);
                if (FAR) {
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const cplx t = cmul(ik, v[d]);
                            const cplx u = {t.re - xp[j][d] * dv.re, t.im - xp[j][d] * dv.im};
                            const cplx r = cmul(kv, u);
                            ar[j][d] += r.re;
                            ai[j][d] += r.im;
                        }
                    } else {
                        const cplx kik = cmul(kv, ik);
                        cplx val[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d) val[d] = cmul(kik, v[d]);
                        const double *x = xp[j];
                        ar[j][0] += x[1] * val[2].re - x[2] * val[1].re;
                        ai[j][0] += x[1] * val[2].im - x[2] * val[1].im;
                        ar[j][1] += x[2] * val[0].re - x[0] * val[2].re;
                        ai[j][1] += x[2] * val[0].im - x[0] * val[2].im;
                        ar[j][2] += x[0] * val[1].re - x[1] * val[0].re;
                        ai[j][2] += x[0] * val[1].im - x[1] * val[0].im;
                    }
                } else {
                    const double df[3] = {xp[j][0] - y[0], xp[j][1] - y[1], xp[j][2] - y[2]};
                    const double dist2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
                    const double dist = sqrt(dist2);
                    const cplx ikd1 = {-ki * dist - 1.0, kr * dist};  // i k dist - 1
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
                        // (i k d - 1) dv / (i k d^2)
                        const cplx ikd2 = {-ki * dist2, kr * dist2};
                        const double den = ikd2.re * ikd2.re + ikd2.im * ikd2.im;
                        const cplx num = cmul(ikd1, dv);
                        const cplx q = {(num.re * ikd2.re + num.im * ikd2.im) / den,
                                        (num.im * ikd2.re - num.re * ikd2.im) / den};
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const cplx t = cmul(ik, v[d]);
                            const cplx u = {t.re - df[d] * q.re, t.im - df[d] * q.im};
                            const cplx r = cmul(kv, u);
                            ar[j][d] += r.re;
                            ai[j][d] += r.im;
                        }
                    } else {
                        const cplx f = cscale(cmul(kv, ikd1), 1.0 / dist2);
                        cplx val[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d) val[d] = cmul(f, v[d]);
                        ar[j][0] += df[1] * val[2].re - df[2] * val[1].re;
                        ai[j][0] += df[1] * val[2].im - df[2] * val[1].im;
                        ar[j][1] += df[2] * val[0].re - df[0] * val[2].re;
                        ai[j][1] += df[2] * val[0].im - df[0] * val[2].im;
                        ar[j][2] += df[0] * val[1].re - df[1] * val[0].re;
                        ai[j][2] += df[0] * val[1].im - df[1] * val[0].im;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j)
#pragma unroll
        for (int d = 0; d < KD; ++d) {
            ar[j][d] = warp_sum(ar[j][d]);
            ai[j][d] = warp_sum(ai[j][d]);
        }
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < POT_PPW; ++j) {
            const int64_t pj = p0 + j;
            if (pj >= prm.npoints) break;
#pragma unroll
            for (int d = 0; d < KD; ++d) {
                prm.result[2 * (d * prm.npoints + pj)] = ar[j][d];
                prm.result[2 * (d * prm.npoints + pj) + 1] = ai[j][d];
            }
        }
    }
}

template <int ASM, int K>
static cudaError_t launch_pot(const PotParams &prm, cudaStream_t st) {
    const int64_t warps = (prm.npoints + POT_PPW - 1) / POT_PPW;
    const unsigned blocks = (unsigned)((warps + POT_WARPS - 1) / POT_WARPS);
    potential_eval<ASM, K><<<blocks, 32 * POT_WARPS, 0, st>>>(prm);
    return cudaGetLastError();
}


// ---------------------------------------------------------------------------
// Scalar Laplace / Helmholtz potentials, a thread per evaluation point.
//
// Each thread owns PS_PPT points and walks the sources of its chunk, which the
// block stages in shared memory PS_SOURCES at a time and reads back as
// broadcasts.  The grid is (point blocks, source chunks): ten thousand points
// make only a few dozen blocks of 256 points, so the support is split into
// chunks of whole elements, as many as fill the SMs' resident CTA slots in
// whole waves (scalar_grid), and the chunks' partial sums are added into the
// zeroed result with FP64 atomics (a single chunk stores directly).
//
// Helmholtz phase (real k): for a source y of element e with centroid c_e,
//   k |x - y| = k |x - c_e| + k (|x - y| - |x - c_e|),
// where |x - y| - |x - c_e| is at most |y - c_e| <= R, the grid's largest
// centroid-to-vertex distance.  With k R <= 1/2 (PHC 2) or <= 1 (PHC 1) the
// second part needs no range reduction (sincos_half64 / sincos_small64); the
// element's partial sum is rotated once by exp(i k |x - c_e|) (sincos_cw64).
// PHC 0 reduces the full phase per source.
constexpr int PS_THREADS = 128;
constexpr int PS_PPT = 2;
constexpr int PS_SOURCES = 384;
constexpr int PS_CHUNK_MIN = 16;  // fewest elements in a source chunk

template <int PHC>
__device__ __forceinline__ void phase_small(double t, double *s, double *c) {
    if (PHC == 2)
        sincos_half64(t, s, c);
    else if (PHC == 1)
        sincos_small64(t, s, c);
    else
        sincos_cw64(t, s, c);
}

// PHC 0-2: real wavenumber (1, 2: factored about the element centroid); PHC 3: complex wavenumber
// k = kr + i ki, exp(i kr r) exp(-ki r) per point-source pair and (ikr - 1) = -(1 + ki r) + i kr r.
// Modified Helmholtz (real kernel, w = p[0]): the Laplace kernels times exp(-w r) or exp(-w r) (1 + w r).
template <int K, int PHC, int NQ>
__global__ void __launch_bounds__(PS_THREADS) potential_scalar(PotParams prm, int64_t chunk_elems) {
    constexpr bool HELM = (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP);
    constexpr bool MH = (K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP);
    constexpr bool DLP = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_MODHELM_DLP);
    constexpr bool FACTOR = HELM && (PHC == 1 || PHC == 2);
    constexpr bool CK = HELM && PHC == 3;
    __shared__ double2 ssrc[PS_SOURCES * 4];        // {y0 y1} {y2 cre} {cim n0} {n1 n2}
    __shared__ double2 scen[FACTOR ? PS_SOURCES * 2 : 2];  // {c0 c1} {c2 -} per element
    const int nq = NQ ? NQ : prm.nq;
    const int tile_elems = PS_SOURCES / nq;
    const int64_t ebeg = (int64_t)blockIdx.y * chunk_elems;
    const int64_t eend = min(ebeg + chunk_elems, prm.nsupport);
    const int64_t pbase = (int64_t)blockIdx.x * (PS_THREADS * PS_PPT) + threadIdx.x;
    double x[PS_PPT][3], ar[PS_PPT], ai[PS_PPT];
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = min(pbase + j * PS_THREADS, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[j][d] = prm.points[3 * pj + d];
        ar[j] = ai[j] = 0.0;
    }
    const double k = prm.p[0], ki = CK ? prm.p[1] : 0.0;
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t t0 = ebeg; t0 < eend; t0 += tile_elems) {
        const int te = (int)min((int64_t)tile_elems, eend - t0);
        const int ns = te * nq;
        const int64_t s0 = t0 * nq;
        __syncthreads();
        for (int s = threadIdx.x; s < ns; s += PS_THREADS) {
            const int64_t gs = s0 + s;
            ssrc[4 * s + 0] = make_double2(o[gs], o[n + gs]);
            ssrc[4 * s + 1] = make_double2(o[2 * n + gs], o[6 * n + gs]);
            ssrc[4 * s + 2] = make_double2(o[7 * n + gs], DLP ? o[3 * n + gs] : 0.0);
            if (DLP) ssrc[4 * s + 3] = make_double2(o[4 * n + gs], o[5 * n + gs]);
        }
        if (FACTOR) {
            for (int e = threadIdx.x; e < te; e += PS_THREADS) {
                const int64_t ge = t0 + e;
                scen[2 * e] = make_double2(o[8 * n + ge], o[9 * n + ge]);
                scen[2 * e + 1] = make_double2(o[10 * n + ge], 0.0);
            }
        }
        __syncthreads();
        for (int e = 0; e < te; ++e) {
            double krc[PS_PPT], er[PS_PPT], ei[PS_PPT];
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                krc[j] = 0.0;
                if (FACTOR) {
                    const double2 c01 = scen[2 * e], c2 = scen[2 * e + 1];
                    const double d0 = c01.x - x[j][0], d1 = c01.y - x[j][1], d2 = c2.x - x[j][2];
                    const double rc2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                    krc[j] = rc2 > 0.0 ? k * (rc2 * rsqrt64(rc2)) : 0.0;  // a point may sit on a centroid
                }
                er[j] = ei[j] = 0.0;
            }
#pragma unroll 6
            for (int q = 0; q < nq; ++q) {
                const int s = e * nq + q;
                const double2 y01 = ssrc[4 * s], y2c = ssrc[4 * s + 1], cin = ssrc[4 * s + 2];
                double2 n12 = make_double2(0.0, 0.0);
                if (DLP) n12 = ssrc[4 * s + 3];
                const double cr = y2c.y, ci = cin.x;
#pragma unroll
                for (int j = 0; j < PS_PPT; ++j) {
                    const double d0 = y01.x - x[j][0], d1 = y01.y - x[j][1], d2 = y2c.x - x[j][2];
                    const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                    const double rinv = rsqrt64(r2);
                    // f: real factor of the kernel without 1/(4 pi) and phase
                    double f = rinv;
                    if (DLP) {
                        const double dot = fma(d2, n12.y, fma(d1, n12.x, d0 * cin.y));
                        f = dot * rinv * rinv * rinv;
                    }
                    if (!HELM) {
                        if (DLP) f = -f;
                        if (MH) {
                            const double r = r2 * rinv, e = exp(-k * r);
                            f *= DLP ? e * fma(k, r, 1.0) : e;
                        }
                        er[j] = fma(f, cr, er[j]);
                        ei[j] = fma(f, ci, ei[j]);
                    } else {
                        const double r = r2 * rinv;
                        double sn, cs;
                        phase_small<CK ? 0 : PHC>(FACTOR ? fma(k, r, -krc[j]) : k * r, &sn, &cs);
                        if (CK) {
                            const double am = exp(-ki * r);
                            sn *= am;
                            cs *= am;
                        }
                        double wr = f * cr, wi = f * ci;  // f times the coefficient
                        if (DLP) {
                            // times (i k r - 1) = -a + i b, a = 1 + ki r, b = kr r
                            const double b = k * r, a = CK ? fma(ki, r, 1.0) : 1.0;
                            const double tr = -fma(b, wi, a * wr), ti = fma(b, wr, -a * wi);
                            wr = tr;
                            wi = ti;
                        }
                        er[j] = fma(cs, wr, fma(-sn, wi, er[j]));
                        ei[j] = fma(cs, wi, fma(sn, wr, ei[j]));
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                if (FACTOR) {
                    double sn, cs;
                    sincos_cw64(krc[j], &sn, &cs);
                    ar[j] = fma(cs, er[j], fma(-sn, ei[j], ar[j]));
                    ai[j] = fma(cs, ei[j], fma(sn, er[j], ai[j]));
                } else {
                    ar[j] += er[j];
                    ai[j] += ei[j];
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = pbase + j * PS_THREADS;
        if (pj >= prm.npoints) break;
        double *out = prm.result + 2 * pj;
        if (gridDim.y == 1) {
            out[0] = BC_INV_4PI * ar[j];
            out[1] = BC_INV_4PI * ai[j];
        } else {
            atomicAdd(out, BC_INV_4PI * ar[j]);
            atomicAdd(out + 1, BC_INV_4PI * ai[j]);
        }
    }
}

// Mixed precision (FP32 point-source pairs): Laplace, Helmholtz and modified
// Helmholtz single / double layer potentials.  Lengths are in units of
// 1/kappa (kappa = Re k, omega, or 1 for Laplace).  A complex wavenumber
// (CK) adds the amplitude e^{-beta r'}, beta = Im k / Re k, and modified
// Helmholtz has e^{-r'} alone (real kernel): e^{-beta theta} per pair by
// __expf, e^{-beta r_c'} per (point, element) by exp_neg_reduced; the
// double-layer factor (i k r - 1) becomes -(1 + beta r') + i r', and
// -(1 + r') for modified Helmholtz.  Per (evaluation point, source element) in
// FP64: D = kappa c_e - kappa x (one FMA per coordinate, kappa c_e staged),
// r_c' = |D| (FP32 rsqrt, one FP64 Newton step) and the argument reduction of
// exp(i r_c'); per source in FP32:
// yo = kappa (y_q - c_e), |yo|^2 and yo . n_e; per pair in FP32:
//   r'^2 - r_c'^2 = |yo|^2 + 2 D . yo,  theta = (r'^2 - r_c'^2) / (r' + r_c'),
// 1/r' by rsqrt.approx, sin / cos of theta by the fitted polynomials (phase
// class PHC bounds |theta| <= kappa R), and the complex product with the
// source coefficient; the thread's two evaluation points travel together in
// packed f32x2 operations.  The six-term sums per element, exp(i r_c') (FP32
// polynomials after the FP64 reduction, phase_reduced32) and their product are
// FP32; the sum over elements is FP64, in units of kappa (single layer) or
// kappa^2 (double layer), which multiply once at the end.  B200 runs FP64 at
// half the FP32 rate, so every FP64 operation per (point, element) costs about
// as much as the FP32 work of one pair: the FP64 part is kept to ~20 of them.  Single layer e^{ikr}/r = kappa e^{i theta} e^{i r_c'} / r'; double
// layer (ikr - 1) e^{ikr} (d . n) / r^3 = kappa^2 (i r' - 1) e^{i theta}
// e^{i r_c'} (d' . n) / r'^3 with d' = D + yo.
// Near elements: with r_c' >= 4 kappa R (R >= every source's distance from its
// element centroid) the FP32 sums lose at most ~1.6e-7 relative in r'^2; a
// point closer to an element than that (evaluation next to the surface)
// takes that element's sources in FP64 instead (`near_r` = 4 kappa R, 0 when R
// is unknown: no FP64 fallback).
// NQ > 0 fixes the sources per element at compile time (the pair loop unrolls);
// NQ = 0 reads it from prm.nq.
template <int K, int PHC, int NQ, bool CK = false>
__global__ void __launch_bounds__(PS_THREADS) potential_scalar_mixed(PotParams prm, int64_t chunk_elems,
                                                                      double near_r) {
    constexpr bool HELM = (K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP);
    constexpr bool MH = (K == BEMPPCUDA_MODHELM_SLP || K == BEMPPCUDA_MODHELM_DLP);
    constexpr bool DLP = (K == BEMPPCUDA_LAPLACE_DLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_MODHELM_DLP);
    constexpr bool EXPO = MH || CK;  // an amplitude exp(-beta r') beside (or instead of) the phase
    static_assert(!CK || HELM, "complex wavenumber: Helmholtz potentials");
    static_assert(PS_PPT == 2, "two evaluation points per thread, packed");
    __shared__ float4 syo[PS_SOURCES];  // yo, |yo|^2
    __shared__ float4 scf[PS_SOURCES];  // coefficient re, im, yo . n_e, -im
    __shared__ double scen[PS_SOURCES * 3];  // kappa c_e
    __shared__ float snrm[DLP ? PS_SOURCES * 3 : 3];
    const int nq = NQ > 0 ? NQ : prm.nq;
    const int tile_elems = PS_SOURCES / nq;
    const int64_t ebeg = (int64_t)blockIdx.y * chunk_elems;
    const int64_t eend = min(ebeg + chunk_elems, prm.nsupport);
    const int64_t pbase = (int64_t)blockIdx.x * (PS_THREADS * PS_PPT) + threadIdx.x;
    const double kap = HELM || MH ? prm.p[0] : 1.0;
    // exp(-beta r'): beta = Im k / Re k (complex k), 1 (modified Helmholtz, units of 1/omega)
    const double betd = CK ? prm.p[1] / prm.p[0] : (MH ? 1.0 : 0.0);
    const float bet = (float)betd;
    const double sc = HELM || MH ? (DLP ? kap * kap : kap) : 1.0;  // the sums ar, ai are in units of sc
    const double inv_sc = __drcp_rn(sc);
    double x[PS_PPT][3], ar[PS_PPT], ai[PS_PPT];
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = min(pbase + j * PS_THREADS, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[j][d] = prm.points[3 * pj + d];
        ar[j] = ai[j] = 0.0;
    }
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t t0 = ebeg; t0 < eend; t0 += tile_elems) {
        const int te = (int)min((int64_t)tile_elems, eend - t0);
        const int ns = te * nq;
        const int64_t s0 = t0 * nq;
        __syncthreads();
        for (int e = threadIdx.x; e < te; e += PS_THREADS) {
            const int64_t ge = t0 + e;
#pragma unroll
            for (int d = 0; d < 3; ++d) scen[3 * e + d] = kap * o[(8 + d) * n + ge];
            if (DLP)
#pragma unroll
                for (int d = 0; d < 3; ++d) snrm[3 * e + d] = (float)o[(3 + d) * n + ge * nq];
        }
        __syncthreads();
        for (int s = threadIdx.x; s < ns; s += PS_THREADS) {
            const int64_t gs = s0 + s;
            const int e = s / nq;
            const float y0 = (float)fma(kap, o[gs], -scen[3 * e]), y1 = (float)fma(kap, o[n + gs], -scen[3 * e + 1]),
                        y2 = (float)fma(kap, o[2 * n + gs], -scen[3 * e + 2]);
            syo[s] = make_float4(y0, y1, y2, fmaf(y2, y2, fmaf(y1, y1, y0 * y0)));
            float yn = 0.f;
            if (DLP) yn = fmaf(y2, snrm[3 * e + 2], fmaf(y1, snrm[3 * e + 1], y0 * snrm[3 * e]));
            const float cim = (float)o[7 * n + gs];
            scf[s] = make_float4((float)o[6 * n + gs], cim, yn, -cim);
        }
        __syncthreads();
        for (int e = 0; e < te; ++e) {
            // per (point, element): D = kappa (c_e - x) in FP64, packed FP32 copies for the pairs
            double rc[PS_PPT];
            float dd[3][PS_PPT], rc2h[PS_PPT];
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                const double D0 = fma(-kap, x[j][0], scen[3 * e]), D1 = fma(-kap, x[j][1], scen[3 * e + 1]),
                             D2 = fma(-kap, x[j][2], scen[3 * e + 2]);
                const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
                rc2h[j] = (float)rc2;
                // r_c' from the FP32 rsqrt and one FP64 Newton step (relative error ~1e-13); the clamp
                // keeps a point on a centroid (rc2 = 0) at r_c' = 0
                const double y0 = (double)rsqrt_approx(fmaxf(rc2h[j], 1e-30f));
                const double r0 = rc2 * y0;
                rc[j] = fma(r0, 0.5 * fma(-r0, y0, 1.0), r0);
                dd[0][j] = (float)D0;
                dd[1][j] = (float)D1;
                dd[2][j] = (float)D2;
            }
            // D . n_e enters the double layer as a factor (no cancellation): FP32 is enough
            const float2 Dh0 = f2(dd[0][0], dd[0][1]), Dh1 = f2(dd[1][0], dd[1][1]), Dh2 = f2(dd[2][0], dd[2][1]);
            const float2 Dn = DLP ? fma2(Dh2, b2(snrm[3 * e + 2]), fma2(Dh1, b2(snrm[3 * e + 1]),
                                                                       mul2(Dh0, b2(snrm[3 * e]))))
                                  : b2(0.f);
            const float2 Dx = add2(Dh0, Dh0), Dy = add2(Dh1, Dh1), Dz = add2(Dh2, Dh2);  // 2 D
            const float2 rcf = f2((float)rc[0], (float)rc[1]);
            const float2 rc2f = f2(rc2h[0], rc2h[1]);
            float2 er = b2(0.f), ei = b2(0.f);
#pragma unroll(NQ > 0 ? NQ : 1)
            for (int q = 0; q < nq; ++q) {
                const float4 yo = syo[e * nq + q];
                const float4 cf = scf[e * nq + q];
                const float2 sdot = fma2(Dz, b2(yo.z), fma2(Dy, b2(yo.y), fma2(Dx, b2(yo.x), b2(yo.w))));
                const float2 r2 = add2(rc2f, sdot);
                const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                const float2 cr = b2(cf.x), ci = b2(cf.y);
                if (!HELM && !MH) {
                    float2 f = rinv;
                    if (DLP) {
                        // -(d'.n) / r'^3
                        const float2 dot = add2(Dn, b2(cf.z));
                        f = mul2(mul2(rinv, rinv), mul2(rinv, mul2(dot, b2(-1.f))));
                    }
                    er = fma2(f, cr, er);
                    ei = fma2(f, ci, ei);
                } else {
                    const float2 den = fma2(r2, rinv, rcf);  // r' + r_c'
                    const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                    // cs + i sn: e^{i theta} (Helmholtz), times e^{-beta theta} (complex k); e^{-theta} (modified)
                    float2 sn = b2(0.f), cs = b2(1.f);
                    if (HELM) sincos2<PHC>(th, &sn, &cs);
                    if (EXPO) {
                        const float2 am = f2(__expf(-bet * th.x), __expf(-bet * th.y));
                        cs = mul2(cs, am);
                        if (HELM) sn = mul2(sn, am);
                    }
                    // kernel value over kappa (SLP) or kappa^2 (DLP), the element factor e^{(i - beta) r_c'} excluded
                    float2 vr, vi = b2(0.f);
                    if (!DLP) {
                        vr = mul2(rinv, cs);
                        if (HELM) vi = mul2(rinv, sn);
                    } else {
                        const float2 rp = mul2(r2, rinv);
                        const float2 g = mul2(add2(Dn, b2(cf.z)), mul2(rinv, mul2(rinv, rinv)));
                        if (MH) {
                            // -(1 + r') e^{-theta} (d'.n) / r'^3
                            vr = mul2(g, mul2(mul2(add2(rp, b2(1.f)), cs), b2(-1.f)));
                        } else if (CK) {
                            // (i k r - 1) = -(1 + beta r') + i r': (-a cs - r' sn, r' cs - a sn) g
                            const float2 a = fma2(b2(bet), rp, b2(1.f));
                            vr = mul2(g, mul2(fma2(rp, sn, mul2(a, cs)), b2(-1.f)));
                            vi = mul2(g, fma2(rp, cs, mul2(mul2(a, sn), b2(-1.f))));
                        } else {
                            // (i r' - 1) e^{i theta} (d'.n) / r'^3: (-cs - r' sn, r' cs - sn) g
                            vr = mul2(g, mul2(fma2(rp, sn, cs), b2(-1.f)));
                            vi = mul2(g, fma2(rp, cs, mul2(sn, b2(-1.f))));
                        }
                    }
                    if (MH) {  // real kernel
                        er = fma2(vr, cr, er);
                        ei = fma2(vr, ci, ei);
                    } else {
                        er = fma2(vr, cr, fma2(vi, b2(cf.w), er));  // cf.w = -im, exact
                        ei = fma2(vr, ci, fma2(vi, cr, ei));
                    }
                }
            }
            // times exp(i r_c') in packed FP32 (the phase and the sums carry FP32 errors alike); the
            // FP64 sums over elements leave out kappa (single layer) or kappa^2 (double layer)
            float2 pr = er, pi = ei;
            double amp[2] = {1.0, 1.0};  // e^{-beta r_c'} (complex k, modified Helmholtz)
            if (EXPO) {
                amp[0] = exp_neg_reduced(betd * rc[0]);
                amp[1] = exp_neg_reduced(betd * rc[1]);
            }
            if (HELM) {
                float s0f, c0f, s1f, c1f;  // FP64 reduction, FP32 polynomials (phase_reduced32)
                phase_reduced32(rc[0], &s0f, &c0f);
                phase_reduced32(rc[1], &s1f, &c1f);
                const float2 cs = f2(c0f, c1f), sn = f2(s0f, s1f);
                pr = fma2(cs, er, mul2(sn, mul2(ei, b2(-1.f))));
                pi = fma2(cs, ei, mul2(sn, er));
            }
            const double prj[2] = {(double)pr.x, (double)pr.y}, pij[2] = {(double)pi.x, (double)pi.y};
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                if (rc[j] < near_r) {
                    // FP64 for this (point, element): the sources from the table in global memory
                    double nr = 0.0, ni = 0.0;
                    const int64_t g0 = s0 + (int64_t)e * nq;
                    for (int q = 0; q < nq; ++q) {
                        const int64_t gq = g0 + q;
                        const double d0 = o[gq] - x[j][0], d1 = o[n + gq] - x[j][1], d2 = o[2 * n + gq] - x[j][2];
                        const double r2 = fma(d2, d2, fma(d1, d1, d0 * d0));
                        const double rinv = rsqrt64(r2);
                        double f = rinv;
                        if (DLP) f = fma(d2, o[5 * n + gq], fma(d1, o[4 * n + gq], d0 * o[3 * n + gq])) * rinv * rinv * rinv;
                        const double cr = o[6 * n + gq], ci = o[7 * n + gq];
                        if (!HELM && !MH) {
                            if (DLP) f = -f;
                            nr = fma(f, cr, nr);
                            ni = fma(f, ci, ni);
                        } else if (MH) {
                            // the Laplace kernels times e^{-w r} (single layer), e^{-w r} (1 + w r) (double layer)
                            const double r = r2 * rinv;
                            double w = f * exp(-kap * r);
                            if (DLP) w = -w * fma(kap, r, 1.0);
                            nr = fma(w, cr, nr);
                            ni = fma(w, ci, ni);
                        } else {
                            const double r = r2 * rinv;
                            double sn, cs;
                            sincos_cw64(kap * r, &sn, &cs);
                            if (CK) {
                                const double am = exp(-prm.p[1] * r);
                                sn *= am;
                                cs *= am;
                            }
                            double wr = f * cr, wi = f * ci;
                            if (DLP) {  // times (i k r - 1) = -(1 + Im k r) + i Re k r
                                const double b = kap * r, c0 = CK ? -fma(prm.p[1], r, 1.0) : -1.0;
                                const double tr = fma(c0, wr, -b * wi), ti = fma(c0, wi, b * wr);
                                wr = tr;
                                wi = ti;
                            }
                            nr = fma(cs, wr, fma(-sn, wi, nr));
                            ni = fma(cs, wi, fma(sn, wr, ni));
                        }
                    }
                    ar[j] = fma(nr, inv_sc, ar[j]);
                    ai[j] = fma(ni, inv_sc, ai[j]);
                } else if (EXPO) {
                    ar[j] = fma(amp[j], prj[j], ar[j]);
                    ai[j] = fma(amp[j], pij[j], ai[j]);
                } else {
                    ar[j] += prj[j];
                    ai[j] += pij[j];
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = pbase + j * PS_THREADS;
        if (pj >= prm.npoints) break;
        double *out = prm.result + 2 * pj;
        const double scale = BC_INV_4PI * sc;
        if (gridDim.y == 1) {
            out[0] = scale * ar[j];
            out[1] = scale * ai[j];
        } else {
            atomicAdd(out, scale * ar[j]);
            atomicAdd(out + 1, scale * ai[j]);
        }
    }
}

// Mixed-precision scalar far fields (helmholtz_far_field_{single,double}_layer,
// numba_kernels.py:402-449): u(x) = (1/4 pi) sum_y e^{-i k x . y} c_y (single
// layer), each term times -k (x . n_y) i (double layer), for unit directions x
// and k = Re k, as the reference evaluates them.  The phase is split about the
// source's element centroid: per (direction, element) in FP64
// phi = -x . (k c_e) and its reduction (phase_reduced32); per source in FP32
// theta = -x . k (y - c_e), |theta| <= k R (phase class PHC), the fitted sine /
// cosine and the complex product with the coefficient; the thread's two
// directions share each source in packed f32x2 operations.  The six-term sums
// per element are FP32, their product with e^{i phi} too; the sum over
// elements is FP64.  No near field: the kernel is smooth.
template <int K, int PHC, int NQ>
__global__ void __launch_bounds__(PS_THREADS) farfield_scalar_mixed(PotParams prm, int64_t chunk_elems) {
    constexpr bool DLP = K == BEMPPCUDA_FARFIELD_DLP;
    static_assert(PS_PPT == 2, "two directions per thread, packed");
    __shared__ float4 syo[PS_SOURCES];                 // -k (y - c_e)
    __shared__ float4 scf[PS_SOURCES];                 // coefficient re, im, -im
    __shared__ double scen[PS_SOURCES * 3];            // k c_e
    __shared__ float snrm[DLP ? PS_SOURCES * 3 : 3];  // n_e
    const int nq = NQ > 0 ? NQ : prm.nq;
    const int tile_elems = PS_SOURCES / nq;
    const int64_t ebeg = (int64_t)blockIdx.y * chunk_elems;
    const int64_t eend = min(ebeg + chunk_elems, prm.nsupport);
    const int64_t pbase = (int64_t)blockIdx.x * (PS_THREADS * PS_PPT) + threadIdx.x;
    const double kap = prm.p[0];
    double x[PS_PPT][3], ar[PS_PPT], ai[PS_PPT];
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = min(pbase + j * PS_THREADS, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) x[j][d] = prm.points[3 * pj + d];
        ar[j] = ai[j] = 0.0;
    }
    const float2 xx = f2((float)x[0][0], (float)x[1][0]), xy = f2((float)x[0][1], (float)x[1][1]),
                 xz = f2((float)x[0][2], (float)x[1][2]);
    // the phase class bounds |theta| <= k R for unit directions; a longer direction takes the reduced
    // polynomials, which hold for any argument
    const bool unit = fmax(fma(x[0][2], x[0][2], fma(x[0][1], x[0][1], x[0][0] * x[0][0])),
                           fma(x[1][2], x[1][2], fma(x[1][1], x[1][1], x[1][0] * x[1][0]))) <= 1.0 + 1e-6;
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t t0 = ebeg; t0 < eend; t0 += tile_elems) {
        const int te = (int)min((int64_t)tile_elems, eend - t0);
        const int ns = te * nq;
        const int64_t s0 = t0 * nq;
        __syncthreads();
        for (int e = threadIdx.x; e < te; e += PS_THREADS) {
            const int64_t ge = t0 + e;
#pragma unroll
            for (int d = 0; d < 3; ++d) scen[3 * e + d] = kap * o[(8 + d) * n + ge];
            if (DLP)
#pragma unroll
                for (int d = 0; d < 3; ++d) snrm[3 * e + d] = (float)o[(3 + d) * n + ge * nq];
        }
        __syncthreads();
        for (int s = threadIdx.x; s < ns; s += PS_THREADS) {
            const int64_t gs = s0 + s;
            const int e = s / nq;
            syo[s] = make_float4((float)fma(-kap, o[gs], scen[3 * e]), (float)fma(-kap, o[n + gs], scen[3 * e + 1]),
                                 (float)fma(-kap, o[2 * n + gs], scen[3 * e + 2]), 0.f);
            const float cim = (float)o[7 * n + gs];
            scf[s] = make_float4((float)o[6 * n + gs], cim, -cim, 0.f);
        }
        __syncthreads();
        for (int e = 0; e < te; ++e) {
            float2 er = b2(0.f), ei = b2(0.f);
#pragma unroll(NQ > 0 ? NQ : 1)
            for (int q = 0; q < nq; ++q) {
                const float4 yo = syo[e * nq + q];
                const float4 cf = scf[e * nq + q];
                const float2 th = fma2(xz, b2(yo.z), fma2(xy, b2(yo.y), mul2(xx, b2(yo.x))));
                float2 sn, cs;
                if (unit)
                    sincos2<PHC>(th, &sn, &cs);
                else
                    sincos2<0>(th, &sn, &cs);
                const float2 cr = b2(cf.x), ci = b2(cf.y);
                er = fma2(cs, cr, fma2(sn, b2(cf.z), er));  // cf.z = -im, exact
                ei = fma2(cs, ci, fma2(sn, cr, ei));
            }
            // times e^{i phi}, phi = -x . (k c_e): FP64 reduction, FP32 polynomials
            float s0f, c0f, s1f, c1f;
            phase_reduced32(-fma(x[0][2], scen[3 * e + 2], fma(x[0][1], scen[3 * e + 1], x[0][0] * scen[3 * e])),
                            &s0f, &c0f);
            phase_reduced32(-fma(x[1][2], scen[3 * e + 2], fma(x[1][1], scen[3 * e + 1], x[1][0] * scen[3 * e])),
                            &s1f, &c1f);
            const float2 cs = f2(c0f, c1f), sn = f2(s0f, s1f);
            float2 pr = fma2(cs, er, mul2(sn, mul2(ei, b2(-1.f))));
            float2 pi = fma2(cs, ei, mul2(sn, er));
            if (DLP) {
                // times -(x . n_e) i (k applied at the store)
                const float2 f = mul2(fma2(xz, b2(snrm[3 * e + 2]), fma2(xy, b2(snrm[3 * e + 1]),
                                                                       mul2(xx, b2(snrm[3 * e])))), b2(-1.f));
                const float2 tr = mul2(mul2(f, pi), b2(-1.f));
                pi = mul2(f, pr);
                pr = tr;
            }
            ar[0] += (double)pr.x;
            ar[1] += (double)pr.y;
            ai[0] += (double)pi.x;
            ai[1] += (double)pi.y;
        }
    }
    const double scale = BC_INV_4PI * (DLP ? kap : 1.0);
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = pbase + j * PS_THREADS;
        if (pj >= prm.npoints) break;
        double *out = prm.result + 2 * pj;
        if (gridDim.y == 1) {
            out[0] = scale * ar[j];
            out[1] = scale * ai[j];
        } else {
            atomicAdd(out, scale * ar[j]);
            atomicAdd(out + 1, scale * ai[j]);
        }
    }
}

// Mixed-precision Maxwell far fields (maxwell_{e,m}field_far_field, numba_kernels.py:2437-2570): with
// kv = e^{-i k x . y} / (4 pi) (k = Re k in the phase, as potential_eval evaluates it) and per source the
// weighted basis value v (3 complex) and divergence dv,
//   electric: u = i k V - x W,  magnetic: u = i k (x x V),  V = sum_y kv v,  W = sum_y kv dv,
// i k with the complex wavenumber.  V and W are sums of e^{-i k x . y} against per-source coefficients,
// split about the element centroids as in farfield_scalar_mixed: FP64 phase per (direction, element),
// FP32 offsets, polynomials and complex products per source, FP64 sums over elements.
// Only the magnetic field is dispatched here: in W the two triangles of each RWG function add
// divergences of opposite sign, so neighbouring elements' contributions cancel to O(k h) and the FP32
// rounding of each element's sum is amplified by ~1 / (k h) (6e-7 relative at 8192 elements, k = 5,
// growing with refinement); the electric far field stays FP64.
template <int ASM, int PHC, int NQ>
__global__ void __launch_bounds__(PS_THREADS) farfield_maxwell_mixed(PotParams prm, int64_t chunk_elems) {
    constexpr bool EF = ASM == BEMPPCUDA_ASM_EFIE;
    static_assert(PS_PPT == 2, "two directions per thread, packed");
    __shared__ float4 syo[PS_SOURCES];         // -k (y - c_e)
    __shared__ float4 sv01[PS_SOURCES];        // v_0, v_1 (re, im)
    __shared__ float4 sv2d[PS_SOURCES];        // v_2, dv (re, im)
    __shared__ double scen[PS_SOURCES * 3];    // k c_e
    const int nq = NQ > 0 ? NQ : prm.nq;
    const int tile_elems = PS_SOURCES / nq;
    const int64_t ebeg = (int64_t)blockIdx.y * chunk_elems;
    const int64_t eend = min(ebeg + chunk_elems, prm.nsupport);
    const int64_t pbase = (int64_t)blockIdx.x * (PS_THREADS * PS_PPT) + threadIdx.x;
    const double kap = prm.p[0];
    double x[PS_PPT][3], vr[PS_PPT][3], vi[PS_PPT][3], wr[PS_PPT], wi[PS_PPT];
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = min(pbase + j * PS_THREADS, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x[j][d] = prm.points[3 * pj + d];
            vr[j][d] = vi[j][d] = 0.0;
        }
        wr[j] = wi[j] = 0.0;
    }
    const float2 xx = f2((float)x[0][0], (float)x[1][0]), xy = f2((float)x[0][1], (float)x[1][1]),
                 xz = f2((float)x[0][2], (float)x[1][2]);
    // the phase class bounds |theta| <= k R for unit directions; a longer direction takes the reduced
    // polynomials, which hold for any argument
    const bool unit = fmax(fma(x[0][2], x[0][2], fma(x[0][1], x[0][1], x[0][0] * x[0][0])),
                           fma(x[1][2], x[1][2], fma(x[1][1], x[1][1], x[1][0] * x[1][0]))) <= 1.0 + 1e-6;
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t t0 = ebeg; t0 < eend; t0 += tile_elems) {
        const int te = (int)min((int64_t)tile_elems, eend - t0);
        const int ns = te * nq;
        const int64_t s0 = t0 * nq;
        __syncthreads();
        for (int e = threadIdx.x; e < te; e += PS_THREADS) {
            const int64_t el = prm.support[t0 + e];
#pragma unroll
            for (int d = 0; d < 3; ++d) scen[3 * e + d] = kap * __ldg(prm.g + (22 + d) * prm.ne + el);
        }
        __syncthreads();
        for (int s = threadIdx.x; s < ns; s += PS_THREADS) {
            const int64_t gs = s0 + s;
            const int e = s / nq;
            syo[s] = make_float4((float)fma(-kap, o[gs], scen[3 * e]), (float)fma(-kap, o[n + gs], scen[3 * e + 1]),
                                 (float)fma(-kap, o[2 * n + gs], scen[3 * e + 2]), 0.f);
            sv01[s] = make_float4((float)o[6 * n + gs], (float)o[7 * n + gs], (float)o[8 * n + gs],
                                  (float)o[9 * n + gs]);
            sv2d[s] = make_float4((float)o[10 * n + gs], (float)o[11 * n + gs], EF ? (float)o[12 * n + gs] : 0.f,
                                  EF ? (float)o[13 * n + gs] : 0.f);
        }
        __syncthreads();
        for (int e = 0; e < te; ++e) {
            float2 ar[3] = {b2(0.f), b2(0.f), b2(0.f)}, ai[3] = {b2(0.f), b2(0.f), b2(0.f)};
            float2 br = b2(0.f), bi = b2(0.f);
#pragma unroll(NQ > 0 ? NQ : 1)
            for (int q = 0; q < nq; ++q) {
                const float4 yo = syo[e * nq + q];
                const float4 va = sv01[e * nq + q], vb = sv2d[e * nq + q];
                const float2 th = fma2(xz, b2(yo.z), fma2(xy, b2(yo.y), mul2(xx, b2(yo.x))));
                float2 sn, cs;
                if (unit)
                    sincos2<PHC>(th, &sn, &cs);
                else
                    sincos2<0>(th, &sn, &cs);
                const float2 msn = mul2(sn, b2(-1.f));
                const float cre[4] = {va.x, va.z, vb.x, vb.z}, cim[4] = {va.y, va.w, vb.y, vb.w};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    ar[d] = fma2(cs, b2(cre[d]), fma2(msn, b2(cim[d]), ar[d]));
                    ai[d] = fma2(cs, b2(cim[d]), fma2(sn, b2(cre[d]), ai[d]));
                }
                if (EF) {
                    br = fma2(cs, b2(cre[3]), fma2(msn, b2(cim[3]), br));
                    bi = fma2(cs, b2(cim[3]), fma2(sn, b2(cre[3]), bi));
                }
            }
            // times e^{i phi}, phi = -x . (k c_e)
            float s0f, c0f, s1f, c1f;
            phase_reduced32(-fma(x[0][2], scen[3 * e + 2], fma(x[0][1], scen[3 * e + 1], x[0][0] * scen[3 * e])),
                            &s0f, &c0f);
            phase_reduced32(-fma(x[1][2], scen[3 * e + 2], fma(x[1][1], scen[3 * e + 1], x[1][0] * scen[3 * e])),
                            &s1f, &c1f);
            const float2 cs = f2(c0f, c1f), sn = f2(s0f, s1f), msn = mul2(sn, b2(-1.f));
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float2 pr = fma2(cs, ar[d], mul2(msn, ai[d])), pi = fma2(cs, ai[d], mul2(sn, ar[d]));
                vr[0][d] += (double)pr.x;
                vr[1][d] += (double)pr.y;
                vi[0][d] += (double)pi.x;
                vi[1][d] += (double)pi.y;
            }
            if (EF) {
                const float2 pr = fma2(cs, br, mul2(msn, bi)), pi = fma2(cs, bi, mul2(sn, br));
                wr[0] += (double)pr.x;
                wr[1] += (double)pr.y;
                wi[0] += (double)pi.x;
                wi[1] += (double)pi.y;
            }
        }
    }
    // i k with the complex wavenumber, 1 / (4 pi)
    const double ikr = -prm.p[1] * BC_INV_4PI, iki = prm.p[0] * BC_INV_4PI;
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = pbase + j * PS_THREADS;
        if (pj >= prm.npoints) break;
        double ur[3], ui[3];
        if (EF) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ur[d] = ikr * vr[j][d] - iki * vi[j][d] - BC_INV_4PI * x[j][d] * wr[j];
                ui[d] = ikr * vi[j][d] + iki * vr[j][d] - BC_INV_4PI * x[j][d] * wi[j];
            }
        } else {
            double cr[3], ci[3];  // x x V
            cr[0] = x[j][1] * vr[j][2] - x[j][2] * vr[j][1];
            cr[1] = x[j][2] * vr[j][0] - x[j][0] * vr[j][2];
            cr[2] = x[j][0] * vr[j][1] - x[j][1] * vr[j][0];
            ci[0] = x[j][1] * vi[j][2] - x[j][2] * vi[j][1];
            ci[1] = x[j][2] * vi[j][0] - x[j][0] * vi[j][2];
            ci[2] = x[j][0] * vi[j][1] - x[j][1] * vi[j][0];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ur[d] = ikr * cr[d] - iki * ci[d];
                ui[d] = ikr * ci[d] + iki * cr[d];
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double *out = prm.result + 2 * (d * prm.npoints + pj);
            if (gridDim.y == 1) {
                out[0] = ur[d];
                out[1] = ui[d];
            } else {
                atomicAdd(out, ur[d]);
                atomicAdd(out + 1, ui[d]);
            }
        }
    }
}

// Mixed-precision Maxwell magnetic potential (maxwell_mfield_potential, numba_kernels.py:2363-2433):
// H(x) = sum_y G (i k d - 1) / d^2 (x - y) x v_y, d = |x - y|, v the weighted basis values.  In units of
// 1/kappa (kappa = Re k) about the source's element centroid, as potential_scalar_mixed:
//   H = -(kappa^2 / 4 pi) sum_e e^{i r_c'} sum_q h (d' x v),  h = (i r' - 1) e^{i theta} / r'^3,
// d' = kappa (y - x) = D + yo; a complex k adds e^{-beta r'} (beta = Im k / Re k) split the same way and
// (i k d - 1) = -(1 + beta r') + i r'.  Per pair in packed FP32 (the thread's two points): r', theta, h, the
// cross product d' x v and h times it; per (point, element) in FP64: D, r_c', the phase and amplitude and
// the sums over elements.  A point within 4 kappa R of an element takes that element's sources in FP64.
// The electric potential is not done this way: its divergence term cancels between the two triangles of
// each RWG function, which FP32 element sums do not survive (the same reason as the electric far field).
template <int PHC, int NQ, bool CK>
__global__ void __launch_bounds__(PS_THREADS) potential_mfield_mixed(PotParams prm, int64_t chunk_elems,
                                                                     double near_r) {
    static_assert(PS_PPT == 2, "two evaluation points per thread, packed");
    __shared__ float4 syo[PS_SOURCES];       // yo, |yo|^2
    __shared__ float4 sv01[PS_SOURCES];      // v_0, v_1 (re, im)
    __shared__ float2 sv2[PS_SOURCES];       // v_2 (re, im)
    __shared__ double scen[PS_SOURCES * 3];  // kappa c_e
    const int nq = NQ > 0 ? NQ : prm.nq;
    const int tile_elems = PS_SOURCES / nq;
    const int64_t ebeg = (int64_t)blockIdx.y * chunk_elems;
    const int64_t eend = min(ebeg + chunk_elems, prm.nsupport);
    const int64_t pbase = (int64_t)blockIdx.x * (PS_THREADS * PS_PPT) + threadIdx.x;
    const double kap = prm.p[0], ki = CK ? prm.p[1] : 0.0;
    const double betd = CK ? ki / kap : 0.0;
    const float bet = (float)betd;
    double x[PS_PPT][3], hr[PS_PPT][3], hi[PS_PPT][3];  // hr, hi: the sums in units of -kappa^2 / 4 pi
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = min(pbase + j * PS_THREADS, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x[j][d] = prm.points[3 * pj + d];
            hr[j][d] = hi[j][d] = 0.0;
        }
    }
    const double unit = -kap * kap * BC_INV_4PI;  // the sums' unit
    const double inv_unit = 1.0 / unit;
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t t0 = ebeg; t0 < eend; t0 += tile_elems) {
        const int te = (int)min((int64_t)tile_elems, eend - t0);
        const int ns = te * nq;
        const int64_t s0 = t0 * nq;
        __syncthreads();
        for (int e = threadIdx.x; e < te; e += PS_THREADS) {
            const int64_t el = prm.support[t0 + e];
#pragma unroll
            for (int d = 0; d < 3; ++d) scen[3 * e + d] = kap * __ldg(prm.g + (22 + d) * prm.ne + el);
        }
        __syncthreads();
        for (int s = threadIdx.x; s < ns; s += PS_THREADS) {
            const int64_t gs = s0 + s;
            const int e = s / nq;
            const float y0 = (float)fma(kap, o[gs], -scen[3 * e]), y1 = (float)fma(kap, o[n + gs], -scen[3 * e + 1]),
                        y2 = (float)fma(kap, o[2 * n + gs], -scen[3 * e + 2]);
            syo[s] = make_float4(y0, y1, y2, fmaf(y2, y2, fmaf(y1, y1, y0 * y0)));
            sv01[s] = make_float4((float)o[6 * n + gs], (float)o[7 * n + gs], (float)o[8 * n + gs],
                                  (float)o[9 * n + gs]);
            sv2[s] = make_float2((float)o[10 * n + gs], (float)o[11 * n + gs]);
        }
        __syncthreads();
        for (int e = 0; e < te; ++e) {
            double rc[PS_PPT];
            float dd[3][PS_PPT], rc2h[PS_PPT];
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                const double D0 = fma(-kap, x[j][0], scen[3 * e]), D1 = fma(-kap, x[j][1], scen[3 * e + 1]),
                             D2 = fma(-kap, x[j][2], scen[3 * e + 2]);
                const double rc2 = fma(D2, D2, fma(D1, D1, D0 * D0));
                rc2h[j] = (float)rc2;
                const double y0 = (double)rsqrt_approx(fmaxf(rc2h[j], 1e-30f));
                const double r0 = rc2 * y0;
                rc[j] = fma(r0, 0.5 * fma(-r0, y0, 1.0), r0);
                dd[0][j] = (float)D0;
                dd[1][j] = (float)D1;
                dd[2][j] = (float)D2;
            }
            const float2 Dh0 = f2(dd[0][0], dd[0][1]), Dh1 = f2(dd[1][0], dd[1][1]), Dh2 = f2(dd[2][0], dd[2][1]);
            const float2 Dx = add2(Dh0, Dh0), Dy = add2(Dh1, Dh1), Dz = add2(Dh2, Dh2);  // 2 D
            const float2 rcf = f2((float)rc[0], (float)rc[1]);
            const float2 rc2f = f2(rc2h[0], rc2h[1]);
            float2 sr[3] = {b2(0.f), b2(0.f), b2(0.f)}, si[3] = {b2(0.f), b2(0.f), b2(0.f)};
#pragma unroll(NQ > 0 ? NQ : 1)
            for (int q = 0; q < nq; ++q) {
                const float4 yo = syo[e * nq + q];
                const float4 va = sv01[e * nq + q];
                const float2 vb = sv2[e * nq + q];
                const float2 sdot = fma2(Dz, b2(yo.z), fma2(Dy, b2(yo.y), fma2(Dx, b2(yo.x), b2(yo.w))));
                const float2 r2 = add2(rc2f, sdot);
                const float2 rinv = f2(rsqrt_approx(r2.x), rsqrt_approx(r2.y));
                const float2 den = fma2(r2, rinv, rcf);  // r' + r_c'
                const float2 th = mul2(sdot, f2(rcp_approx(den.x), rcp_approx(den.y)));
                float2 sn, cs;
                sincos2<PHC>(th, &sn, &cs);
                if (CK) {
                    const float2 am = f2(__expf(-bet * th.x), __expf(-bet * th.y));
                    cs = mul2(cs, am);
                    sn = mul2(sn, am);
                }
                // h = (i r' - 1) e^{i theta} / r'^3 with a = 1 (+ beta r'): (-(a cs + r' sn), r' cs - a sn) / r'^3
                const float2 rp = mul2(r2, rinv), r3 = mul2(rinv, mul2(rinv, rinv));
                const float2 a = CK ? fma2(b2(bet), rp, b2(1.f)) : b2(1.f);
                const float2 hre = mul2(r3, mul2(fma2(rp, sn, CK ? mul2(a, cs) : cs), b2(-1.f)));
                const float2 him = mul2(r3, fma2(rp, cs, mul2(CK ? mul2(a, sn) : sn, b2(-1.f))));
                // d' = D + yo, then d' x v (real and imaginary parts of v)
                const float2 p0 = add2(Dh0, b2(yo.x)), p1 = add2(Dh1, b2(yo.y)), p2 = add2(Dh2, b2(yo.z));
                const float2 vr0 = b2(va.x), vi0 = b2(va.y), vr1 = b2(va.z), vi1 = b2(va.w), vr2 = b2(vb.x),
                             vi2 = b2(vb.y);
                const float2 cr[3] = {fma2(p1, vr2, mul2(mul2(p2, vr1), b2(-1.f))),
                                      fma2(p2, vr0, mul2(mul2(p0, vr2), b2(-1.f))),
                                      fma2(p0, vr1, mul2(mul2(p1, vr0), b2(-1.f)))};
                const float2 ci[3] = {fma2(p1, vi2, mul2(mul2(p2, vi1), b2(-1.f))),
                                      fma2(p2, vi0, mul2(mul2(p0, vi2), b2(-1.f))),
                                      fma2(p0, vi1, mul2(mul2(p1, vi0), b2(-1.f)))};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    sr[d] = fma2(hre, cr[d], fma2(him, mul2(ci[d], b2(-1.f)), sr[d]));
                    si[d] = fma2(hre, ci[d], fma2(him, cr[d], si[d]));
                }
            }
            // times e^{i r_c'} (and e^{-beta r_c'}), into the FP64 sums; near elements in FP64 instead
            float s0f, c0f, s1f, c1f;
            phase_reduced32(rc[0], &s0f, &c0f);
            phase_reduced32(rc[1], &s1f, &c1f);
            const float2 cs = f2(c0f, c1f), sn = f2(s0f, s1f), msn = mul2(sn, b2(-1.f));
            const double amp[2] = {CK ? exp_neg_reduced(betd * rc[0]) : 1.0, CK ? exp_neg_reduced(betd * rc[1]) : 1.0};
            float2 pr[3], pi[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                pr[d] = fma2(cs, sr[d], mul2(msn, si[d]));
                pi[d] = fma2(cs, si[d], mul2(sn, sr[d]));
            }
#pragma unroll
            for (int j = 0; j < PS_PPT; ++j) {
                if (rc[j] < near_r) {
                    // FP64: sum_q G (i k d - 1) / d^2 (x - y) x v over the element's sources
                    double nr[3] = {0.0, 0.0, 0.0}, ni[3] = {0.0, 0.0, 0.0};
                    const int64_t g0 = s0 + (int64_t)e * nq;
                    for (int q = 0; q < nq; ++q) {
                        const int64_t gq = g0 + q;
                        const double df[3] = {x[j][0] - o[gq], x[j][1] - o[n + gq], x[j][2] - o[2 * n + gq]};
                        const double d2 = fma(df[2], df[2], fma(df[1], df[1], df[0] * df[0]));
                        const double dinv = rsqrt64(d2), dist = d2 * dinv;
                        double snd, csd;
                        sincos_cw64(kap * dist, &snd, &csd);
                        const double am = CK ? exp(-ki * dist) : 1.0;
                        // G (i k d - 1) / d^2 without 1 / (4 pi): e^{ikd} ((-1 - ki d) + i kr d) / d^3
                        const double g3 = am * dinv * dinv * dinv, c0 = -fma(ki, dist, 1.0), c1 = kap * dist;
                        const double fr = g3 * (csd * c0 - snd * c1), fi = g3 * fma(csd, c1, snd * c0);
                        const double vrr[3] = {o[6 * n + gq], o[8 * n + gq], o[10 * n + gq]};
                        const double vii[3] = {o[7 * n + gq], o[9 * n + gq], o[11 * n + gq]};
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const int d1 = (d + 1) % 3, d2i = (d + 2) % 3;
                            const double xr = df[d1] * vrr[d2i] - df[d2i] * vrr[d1];
                            const double xi = df[d1] * vii[d2i] - df[d2i] * vii[d1];
                            nr[d] += fr * xr - fi * xi;
                            ni[d] += fr * xi + fi * xr;
                        }
                    }
                    // into the sums' unit: the FP64 terms lack 1 / (4 pi), the unit is -kappa^2 / (4 pi)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        hr[j][d] = fma(nr[d], BC_INV_4PI * inv_unit, hr[j][d]);
                        hi[j][d] = fma(ni[d], BC_INV_4PI * inv_unit, hi[j][d]);
                    }
                } else {
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        hr[j][d] = fma(amp[j], (double)(j ? pr[d].y : pr[d].x), hr[j][d]);
                        hi[j][d] = fma(amp[j], (double)(j ? pi[d].y : pi[d].x), hi[j][d]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < PS_PPT; ++j) {
        const int64_t pj = pbase + j * PS_THREADS;
        if (pj >= prm.npoints) break;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double *out = prm.result + 2 * (d * prm.npoints + pj);
            if (gridDim.y == 1) {
                out[0] = unit * hr[j][d];
                out[1] = unit * hi[j][d];
            } else {
                atomicAdd(out, unit * hr[j][d]);
                atomicAdd(out + 1, unit * hi[j][d]);
            }
        }
    }
}

// Grid of the per-point kernels: point blocks x source chunks; with more than one chunk the
// chunks add their sums with atomics into the zeroed result.  The chunk count c minimises
//   ceil(pblocks c / slots) (1/c + 1/64),
// slots = SMs x resident CTAs of the kernel being launched (occupancy query): the number of
// waves times the work of one CTA (1/c of its point block's sources) plus a small fixed cost
// per CTA, so that the grid ends on a full wave rather than on a few CTAs of a second one.
static cudaError_t scalar_grid(const PotParams &prm, const void *fn, dim3 *grid, int64_t *chunk_elems,
                               cudaStream_t st, int kdim = 1) {
    int resident = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, fn, PS_THREADS, 0);
    if (err != cudaSuccess) return err;
    const int64_t slots = (int64_t)bc_sm_count() * std::max(resident, 1);
    const int64_t pblocks = (prm.npoints + PS_THREADS * PS_PPT - 1) / (PS_THREADS * PS_PPT);
    int64_t cmax = std::min<int64_t>((prm.nsupport + PS_CHUNK_MIN - 1) / PS_CHUNK_MIN, 65535);
    cmax = std::max<int64_t>(1, std::min<int64_t>(cmax, 8 * ((slots + pblocks - 1) / pblocks)));
    int64_t chunks = 1;
    double best = 0.0;
    for (int64_t c = 1; c <= cmax; ++c) {
        const double t = (double)((pblocks * c + slots - 1) / slots) * (1.0 / (double)c + 1.0 / 64.0);
        if (c == 1 || t < best) {
            best = t;
            chunks = c;
        }
    }
    *chunk_elems = (prm.nsupport + chunks - 1) / chunks;
    chunks = (prm.nsupport + *chunk_elems - 1) / *chunk_elems;
    if (chunks > 1) {
        err = cudaMemsetAsync(prm.result, 0, sizeof(double) * 2 * kdim * prm.npoints, st);
        if (err != cudaSuccess) return err;
    }
    *grid = dim3((unsigned)pblocks, (unsigned)chunks);
    return cudaSuccess;
}

template <int K, int PHC>
static cudaError_t launch_scalar_nq(const PotParams &prm, cudaStream_t st) {
    auto fn = prm.nq == 6 ? potential_scalar<K, PHC, 6> : potential_scalar<K, PHC, 0>;
    dim3 grid;
    int64_t chunk_elems = 0;
    const cudaError_t err = scalar_grid(prm, (const void *)fn, &grid, &chunk_elems, st);
    if (err != cudaSuccess) return err;
    fn<<<grid, PS_THREADS, 0, st>>>(prm, chunk_elems);
    return cudaGetLastError();
}

template <int K, int PHC, bool CK = false>
static cudaError_t launch_mixed_nq(const PotParams &prm, double near_r, cudaStream_t st) {
    auto fn = prm.nq == 6 ? potential_scalar_mixed<K, PHC, 6, CK> : potential_scalar_mixed<K, PHC, 0, CK>;
    dim3 grid;
    int64_t chunk_elems = 0;
    const cudaError_t err = scalar_grid(prm, (const void *)fn, &grid, &chunk_elems, st);
    if (err != cudaSuccess) return err;
    fn<<<grid, PS_THREADS, 0, st>>>(prm, chunk_elems, near_r);
    return cudaGetLastError();
}

// Scalar Laplace, Helmholtz (real or complex wavenumber) and modified Helmholtz potentials;
// phase_radius bounds every source's distance from its element centroid (0: unknown).
// Mixed-precision Laplace, Helmholtz (Re k > 0, real or complex k) and modified Helmholtz single / double
// layer potentials.
template <int K, int PHC>
static cudaError_t launch_far_mixed_nq(const PotParams &prm, cudaStream_t st) {
    auto fn = prm.nq == 6 ? farfield_scalar_mixed<K, PHC, 6> : farfield_scalar_mixed<K, PHC, 0>;
    dim3 grid;
    int64_t chunk_elems = 0;
    const cudaError_t err = scalar_grid(prm, (const void *)fn, &grid, &chunk_elems, st);
    if (err != cudaSuccess) return err;
    fn<<<grid, PS_THREADS, 0, st>>>(prm, chunk_elems);
    return cudaGetLastError();
}

template <int ASM, int PHC>
static cudaError_t launch_far_maxwell_nq(const PotParams &prm, cudaStream_t st) {
    auto fn = prm.nq == 6 ? farfield_maxwell_mixed<ASM, PHC, 6> : farfield_maxwell_mixed<ASM, PHC, 0>;
    dim3 grid;
    int64_t chunk_elems = 0;
    const cudaError_t err = scalar_grid(prm, (const void *)fn, &grid, &chunk_elems, st, 3);
    if (err != cudaSuccess) return err;
    fn<<<grid, PS_THREADS, 0, st>>>(prm, chunk_elems);
    return cudaGetLastError();
}

template <int PHC, bool CK>
static cudaError_t launch_mfield_nq(const PotParams &prm, double near_r, cudaStream_t st) {
    auto fn = prm.nq == 6 ? potential_mfield_mixed<PHC, 6, CK> : potential_mfield_mixed<PHC, 0, CK>;
    dim3 grid;
    int64_t chunk_elems = 0;
    const cudaError_t err = scalar_grid(prm, (const void *)fn, &grid, &chunk_elems, st, 3);
    if (err != cudaSuccess) return err;
    fn<<<grid, PS_THREADS, 0, st>>>(prm, chunk_elems, near_r);
    return cudaGetLastError();
}

// Mixed-precision Maxwell magnetic potential (real or complex k, Re k > 0).
static cudaError_t launch_mfield_mixed(const PotParams &prm, double phase_radius, cudaStream_t st) {
    const double kr = fabs(prm.p[0]) * phase_radius;
    const int phc = (phase_radius > 0.0 && kr <= 0.5) ? 2 : (phase_radius > 0.0 && kr <= 1.0) ? 1 : 0;
    const double near_r = 4.0 * prm.p[0] * phase_radius;  // units of 1 / Re k
    if (prm.p[1] != 0.0) {
        if (phc == 2) return launch_mfield_nq<2, true>(prm, near_r, st);
        if (phc == 1) return launch_mfield_nq<1, true>(prm, near_r, st);
        return launch_mfield_nq<0, true>(prm, near_r, st);
    }
    if (phc == 2) return launch_mfield_nq<2, false>(prm, near_r, st);
    if (phc == 1) return launch_mfield_nq<1, false>(prm, near_r, st);
    return launch_mfield_nq<0, false>(prm, near_r, st);
}

// Mixed-precision Maxwell magnetic far field (the electric one stays FP64: farfield_maxwell_mixed).
static cudaError_t launch_far_maxwell(const PotParams &prm, double phase_radius, cudaStream_t st) {
    const double kr = fabs(prm.p[0]) * phase_radius;
    const int phc = (phase_radius > 0.0 && kr <= 0.5) ? 2 : (phase_radius > 0.0 && kr <= 1.0) ? 1 : 0;
    if (phc == 2) return launch_far_maxwell_nq<BEMPPCUDA_ASM_MFIE, 2>(prm, st);
    if (phc == 1) return launch_far_maxwell_nq<BEMPPCUDA_ASM_MFIE, 1>(prm, st);
    return launch_far_maxwell_nq<BEMPPCUDA_ASM_MFIE, 0>(prm, st);
}

template <int K>
static cudaError_t launch_far_mixed(const PotParams &prm, int phc, cudaStream_t st) {
    if (phc == 2) return launch_far_mixed_nq<K, 2>(prm, st);
    if (phc == 1) return launch_far_mixed_nq<K, 1>(prm, st);
    return launch_far_mixed_nq<K, 0>(prm, st);
}

template <int K, bool CK>
static cudaError_t launch_mixed_phase(const PotParams &prm, int phc, double near_r, cudaStream_t st) {
    if (phc == 2) return launch_mixed_nq<K, 2, CK>(prm, near_r, st);
    if (phc == 1) return launch_mixed_nq<K, 1, CK>(prm, near_r, st);
    return launch_mixed_nq<K, 0, CK>(prm, near_r, st);
}

static cudaError_t launch_scalar_mixed(const PotParams &prm, int kernel, double phase_radius, cudaStream_t st) {
    const double kr = fabs(prm.p[0]) * phase_radius;
    const int phc = (phase_radius > 0.0 && kr <= 0.5) ? 2 : (phase_radius > 0.0 && kr <= 1.0) ? 1 : 0;
    const bool scaled = kernel == BEMPPCUDA_HELMHOLTZ_SLP || kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
                        kernel == BEMPPCUDA_MODHELM_SLP || kernel == BEMPPCUDA_MODHELM_DLP;
    const double near_r = 4.0 * (scaled ? prm.p[0] : 1.0) * phase_radius;  // in the kernel's units of 1/kappa
    const bool ck = prm.p[1] != 0.0;
    switch (kernel) {
    case BEMPPCUDA_FARFIELD_SLP: return launch_far_mixed<BEMPPCUDA_FARFIELD_SLP>(prm, phc, st);
    case BEMPPCUDA_FARFIELD_DLP: return launch_far_mixed<BEMPPCUDA_FARFIELD_DLP>(prm, phc, st);
    case BEMPPCUDA_LAPLACE_SLP: return launch_mixed_nq<BEMPPCUDA_LAPLACE_SLP, 0>(prm, near_r, st);
    case BEMPPCUDA_LAPLACE_DLP: return launch_mixed_nq<BEMPPCUDA_LAPLACE_DLP, 0>(prm, near_r, st);
    case BEMPPCUDA_MODHELM_SLP: return launch_mixed_nq<BEMPPCUDA_MODHELM_SLP, 0>(prm, near_r, st);
    case BEMPPCUDA_MODHELM_DLP: return launch_mixed_nq<BEMPPCUDA_MODHELM_DLP, 0>(prm, near_r, st);
    case BEMPPCUDA_HELMHOLTZ_SLP:
        return ck ? launch_mixed_phase<BEMPPCUDA_HELMHOLTZ_SLP, true>(prm, phc, near_r, st)
                  : launch_mixed_phase<BEMPPCUDA_HELMHOLTZ_SLP, false>(prm, phc, near_r, st);
    default:  // BEMPPCUDA_HELMHOLTZ_DLP
        return ck ? launch_mixed_phase<BEMPPCUDA_HELMHOLTZ_DLP, true>(prm, phc, near_r, st)
                  : launch_mixed_phase<BEMPPCUDA_HELMHOLTZ_DLP, false>(prm, phc, near_r, st);
    }
}

static cudaError_t launch_scalar(const PotParams &prm, int kernel, double phase_radius, cudaStream_t st) {
    const double kr = fabs(prm.p[0]) * phase_radius;
    const int phc = prm.p[1] != 0.0 ? 3
                    : (phase_radius > 0.0 && kr <= 0.5) ? 2 : (phase_radius > 0.0 && kr <= 1.0) ? 1 : 0;
    switch (kernel) {
    case BEMPPCUDA_LAPLACE_SLP: return launch_scalar_nq<BEMPPCUDA_LAPLACE_SLP, 0>(prm, st);
    case BEMPPCUDA_LAPLACE_DLP: return launch_scalar_nq<BEMPPCUDA_LAPLACE_DLP, 0>(prm, st);
    case BEMPPCUDA_MODHELM_SLP: return launch_scalar_nq<BEMPPCUDA_MODHELM_SLP, 0>(prm, st);
    case BEMPPCUDA_MODHELM_DLP: return launch_scalar_nq<BEMPPCUDA_MODHELM_DLP, 0>(prm, st);
    case BEMPPCUDA_HELMHOLTZ_SLP:
        if (phc == 3) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_SLP, 3>(prm, st);
        if (phc == 2) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_SLP, 2>(prm, st);
        if (phc == 1) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_SLP, 1>(prm, st);
        return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_SLP, 0>(prm, st);
    default:  // BEMPPCUDA_HELMHOLTZ_DLP
        if (phc == 3) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_DLP, 3>(prm, st);
        if (phc == 2) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_DLP, 2>(prm, st);
        if (phc == 1) return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_DLP, 1>(prm, st);
        return launch_scalar_nq<BEMPPCUDA_HELMHOLTZ_DLP, 0>(prm, st);
    }
}

}  // namespace bc

using namespace bc;

// Doubles of the source table, or -1 when nsupport * nq * SRC_FIELDS does not fit in int64.
int64_t bc_potential_workspace_doubles(int64_t nsupport, int nq) {
    if (nsupport < 0 || nq < 1 || nsupport > INT64_MAX / ((int64_t)SRC_FIELDS * nq)) return -1;
    return (int64_t)SRC_FIELDS * nsupport * nq;
}

// `workspace` must hold bc_potential_workspace_doubles() doubles.
int bc_potential_launch(const bemppcuda_potential_args *a, double *workspace, cudaStream_t st) {
    PotParams prm;
    prm.g = a->grid.geom;
    prm.ne = a->grid.nelements;
    prm.support = a->space.support;
    prm.nsupport = a->space.nsupport;
    prm.nm = a->space.normal_mult;
    prm.nshape = a->space.nshape;
    prm.nq = a->nq;
    prm.coeff = a->coefficients;
    prm.src = workspace;
    prm.nsrc = a->space.nsupport * a->nq;
    prm.points = a->points;
    prm.npoints = a->npoints;
    prm.result = reinterpret_cast<double *>(a->result);
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    QuadRule rule;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);
    const bool maxwell = a->assembly != BEMPPCUDA_ASM_SCALAR;
    // mixed precision: Laplace, Helmholtz (Re k > 0) and modified Helmholtz (w > 0) single / double layer
    // potentials
    const bool mixed = a->precision == BEMPPCUDA_MIXED;
    if (a->precision != BEMPPCUDA_FP64 && !mixed) {
        bc_set_error("potential: precision must be BEMPPCUDA_FP64 or BEMPPCUDA_MIXED");
        return BEMPPCUDA_ERR_INVALID;
    }
    const bool mixed_kernel =
        a->kernel == BEMPPCUDA_LAPLACE_SLP || a->kernel == BEMPPCUDA_LAPLACE_DLP ||
        ((a->kernel == BEMPPCUDA_HELMHOLTZ_SLP || a->kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
          a->kernel == BEMPPCUDA_MODHELM_SLP || a->kernel == BEMPPCUDA_MODHELM_DLP ||
          a->kernel == BEMPPCUDA_FARFIELD_SLP || a->kernel == BEMPPCUDA_FARFIELD_DLP) &&
         a->params[0] > 0.0);
    // Maxwell: the magnetic potential and far field (the electric ones' divergence sums cancel between
    // neighbouring elements, which FP32 element sums do not survive; farfield_maxwell_mixed)
    const bool maxwell_far = maxwell && a->assembly == BEMPPCUDA_ASM_MFIE &&
                             (a->kernel == BEMPPCUDA_FARFIELD_SLP || a->kernel == BEMPPCUDA_HELMHOLTZ_SLP) &&
                             a->params[0] > 0.0;
    if (mixed && (maxwell ? !maxwell_far : !mixed_kernel)) {
        bc_set_error("mixed-precision potentials: Laplace, Helmholtz (Re k > 0) and modified Helmholtz (w > 0) "
                     "single / double layer potentials, Helmholtz far fields, the Maxwell magnetic potential and far "
                     "field (Re k > 0) only");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    // the FP64 treatment of points next to the surface needs the bound R on source offsets
    if (mixed && !(a->phase_radius > 0.0)) {
        bc_set_error("mixed-precision potentials need phase_radius > 0 (the largest centroid-to-vertex distance "
                     "of the grid): points near the surface take FP64 sources within 4 k R of an element");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (prm.npoints == 0) return BEMPPCUDA_OK;
    if (prm.nsrc > 0) {
        const unsigned blocks = (unsigned)((prm.nsrc + 255) / 256);
        if (maxwell)
            potential_sources<true><<<blocks, 256, 0, st>>>(prm, rule);
        else
            potential_sources<false><<<blocks, 256, 0, st>>>(prm, rule);
    }
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        const bool per_point = a->kernel == BEMPPCUDA_LAPLACE_SLP || a->kernel == BEMPPCUDA_LAPLACE_DLP ||
                               a->kernel == BEMPPCUDA_HELMHOLTZ_SLP || a->kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
                               a->kernel == BEMPPCUDA_MODHELM_SLP || a->kernel == BEMPPCUDA_MODHELM_DLP;
        if (mixed && maxwell && prm.nsupport > 0) {
            err = a->kernel == BEMPPCUDA_FARFIELD_SLP ? launch_far_maxwell(prm, a->phase_radius, st)
                                                      : launch_mfield_mixed(prm, a->phase_radius, st);
        } else if (mixed && prm.nsupport > 0) {
            err = launch_scalar_mixed(prm, a->kernel, a->phase_radius, st);
        } else if (!maxwell && per_point && prm.nsupport > 0) {
            err = launch_scalar(prm, a->kernel, a->phase_radius, st);
        } else if (!maxwell) {
            switch (a->kernel) {
            case BEMPPCUDA_LAPLACE_SLP: err = launch_pot<0, BEMPPCUDA_LAPLACE_SLP>(prm, st); break;
            case BEMPPCUDA_LAPLACE_DLP: err = launch_pot<0, BEMPPCUDA_LAPLACE_DLP>(prm, st); break;
            case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_pot<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
            case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_pot<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, st); break;
            case BEMPPCUDA_MODHELM_SLP: err = launch_pot<0, BEMPPCUDA_MODHELM_SLP>(prm, st); break;
            case BEMPPCUDA_MODHELM_DLP: err = launch_pot<0, BEMPPCUDA_MODHELM_DLP>(prm, st); break;
            case BEMPPCUDA_FARFIELD_SLP: err = launch_pot<0, BEMPPCUDA_FARFIELD_SLP>(prm, st); break;
            case BEMPPCUDA_FARFIELD_DLP: err = launch_pot<0, BEMPPCUDA_FARFIELD_DLP>(prm, st); break;
            default: bc_set_error("kernel %d not valid for a scalar potential", a->kernel); return BEMPPCUDA_ERR_INVALID;
            }
        } else {
            const bool far = a->kernel == BEMPPCUDA_FARFIELD_SLP;
            if (a->kernel != BEMPPCUDA_HELMHOLTZ_SLP && !far) {
                bc_set_error("Maxwell potentials use the Helmholtz single-layer kernel (got %d)", a->kernel);
                return BEMPPCUDA_ERR_INVALID;
            }
            if (a->assembly == BEMPPCUDA_ASM_EFIE)
                err = far ? launch_pot<4, BEMPPCUDA_FARFIELD_SLP>(prm, st) : launch_pot<4, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st);
            else if (a->assembly == BEMPPCUDA_ASM_MFIE)
                err = far ? launch_pot<5, BEMPPCUDA_FARFIELD_SLP>(prm, st) : launch_pot<5, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st);
            else {
                bc_set_error("assembly type %d not valid for a potential", a->assembly);
                return BEMPPCUDA_ERR_INVALID;
            }
        }
    }
    if (err != cudaSuccess) {
        bc_set_error("potential launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
