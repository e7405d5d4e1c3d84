// Singular (Sauter-Schwab) quadrature for coincident, edge-adjacent and
// vertex-adjacent element pairs.
//
// Replaces default_scalar_singular_kernel (numba_kernels.py:1471-1526),
// laplace/helmholtz/modified hypersingular_singular (:1530-1784) and
// maxwell_efield_singular / maxwell_mfield_singular (:1973-2147).
//
// One warp per pair: the lanes stride over the pair's 512-1536 quadrature
// points (coalesced reads of the point and weight tables), accumulate the
// nshape x nshape local block in registers and combine it with xor-shuffle
// reductions.  Always FP64.  Output either to the flat per-pair value array
// of the reference interface or scattered straight into a dense matrix.
#include "common.cuh"
#include "rwg.cuh"  // efie_block
#include "singular_dp0.cuh"

namespace bc {

struct SingParams {
    const double *g;
    int64_t ne;
    const uint32_t *te, *se, *toff, *soff, *woff, *npts;
    const double *tp, *sp, *w;
    int64_t npairs;
    const int32_t *tnm, *snm;
    int nt, ns;
    int is_complex;
    int pad;
    double p[4];
    void *values;
    void *dense;
    int64_t ld;
    const uint32_t *tl2g, *sl2g;
    const double *tmult, *smult;
    double diag_shift;
    int64_t ntab, nw;  // point-table and weight-table lengths
    int64_t mirror_woff;  // > 0: pairs with this weights offset add both orders (test < trial) or nothing
};

// A pair whose element ids or table ranges fall outside the grid / tables is
// skipped (caller-supplied tables are not trusted to be in range).
__device__ __forceinline__ bool pair_in_range(const SingParams &prm, int64_t k) {
    const int64_t t = prm.te[k], s = prm.se[k], n = prm.npts[k];
    const int64_t toff = prm.toff[k], soff = prm.soff[k], woff = prm.woff[k];
    return t >= 0 && t < prm.ne && s >= 0 && s < prm.ne && n >= 0 && toff >= 0 && soff >= 0 && woff >= 0 &&
           toff + n <= prm.ntab && soff + n <= prm.ntab && woff + n <= prm.nw;
}

constexpr int SING_WARPS = 4;  // pairs per block: 128 threads let 3-5 blocks share an SM at 80-170 registers

template <int ASM, int K>
__global__ void __launch_bounds__(32 * SING_WARPS) singular_pairs(SingParams prm) {
    const int lane = threadIdx.x & 31;
    const int64_t k = (int64_t)blockIdx.x * SING_WARPS + (threadIdx.x >> 5);
    if (k >= prm.npairs || !pair_in_range(prm, k)) return;
    const int64_t t = prm.te[k], s = prm.se[k];
    Geom gt, gs;
    load_geom(prm.g, prm.ne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
    load_geom(prm.g, prm.ne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int nt = prm.nt, ns = prm.ns;
    constexpr bool HYP = (ASM == BEMPPCUDA_ASM_LAPLACE_HYP || ASM == BEMPPCUDA_ASM_HELM_HYP ||
                          ASM == BEMPPCUDA_ASM_MODHELM_HYP);
    constexpr bool MAXWELL = (ASM == BEMPPCUDA_ASM_EFIE || ASM == BEMPPCUDA_ASM_MFIE);
    double cp[3][3];
    if (HYP) {
        double ct[3][3], cs[3][3];
        surface_curls(prm.g, prm.ne, t, gt.n, ct);
        surface_curls(prm.g, prm.ne, s, gs.n, cs);
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) cp[i][j] = ct[i][0] * cs[j][0] + ct[i][1] * cs[j][1] + ct[i][2] * cs[j][2];
    }
    const double normal_prod = gt.n[0] * gs.n[0] + gt.n[1] * gs.n[1] + gt.n[2] * gs.n[2];
    const double kr = prm.p[0], ki = prm.p[1];

    double are[3][3], aim[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) are[i][j] = aim[i][j] = 0.0;
    double sre = 0.0, sim = 0.0;  // Helmholtz / modified hypersingular: S = sum_p w G
    // MFIE: the four sums of the pair (MFIE block of rwg.cuh)
    double pbr = 0.0, pbi = 0.0, pcr[3] = {0.0, 0.0, 0.0}, pci[3] = {0.0, 0.0, 0.0};
    double qbr[3] = {0.0, 0.0, 0.0}, qbi[3] = {0.0, 0.0, 0.0}, qcr[3] = {0.0, 0.0, 0.0}, qci[3] = {0.0, 0.0, 0.0};

    const int64_t toff = prm.toff[k], soff = prm.soff[k], woff = prm.woff[k];
    const int n = (int)prm.npts[k];
    for (int m = lane; m < n; m += 32) {
        const double2 tpm = reinterpret_cast<const double2 *>(prm.tp)[toff + m];
        const double2 spm = reinterpret_cast<const double2 *>(prm.sp)[soff + m];
        const double w = __ldg(prm.w + woff + m);
        double x[3], y[3];
        to_global(gt, tpm.x, tpm.y, x);
        to_global(gs, spm.x, spm.y, y);
        const cplx kv = greens<K>(x, y, gt.n, gs.n, prm.p);
        double pt[3], ps[3];
        scalar_shape(nt, tpm.x, tpm.y, pt);
        scalar_shape(ns, spm.x, spm.y, ps);
        if (ASM == BEMPPCUDA_ASM_SCALAR) {
            const cplx kw = cscale(kv, w);
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    if (i < nt && j < ns) {
                        const double f = pt[i] * ps[j];
                        are[i][j] = fma(kw.re, f, are[i][j]);
                        aim[i][j] = fma(kw.im, f, aim[i][j]);
                    }
        } else if (ASM == BEMPPCUDA_ASM_LAPLACE_HYP) {
            are[0][0] = fma(kv.re, w, are[0][0]);
        } else if (HYP) {
            // the pair's value is curl_i.curl_j S + c (n_t.n_s) M_ij with S = sum_p w G and
            // M_ij = sum_p w G phi_i psi_j (the curls and normals are constant per element pair)
            const cplx kw = cscale(kv, w);
            sre += kw.re;
            sim += kw.im;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    if (i < nt && j < ns) {
                        const double f = pt[i] * ps[j];
                        are[i][j] = fma(kw.re, f, are[i][j]);
                        aim[i][j] = fma(kw.im, f, aim[i][j]);
                    }
        } else {
            double bt[3][3], bs[3][3];
            rwg_values(gt, tpm.x, tpm.y, bt);
            rwg_values(gs, spm.x, spm.y, bs);
            const cplx kw = cscale(kv, w);
            if (ASM == BEMPPCUDA_ASM_EFIE) {
                // moments M[a][b] = sum w G u_a(x) v_b(y), u, v = (1, xi, eta): the EFIE block follows per pair
                const double ut[3] = {1.0, tpm.x, tpm.y}, vs[3] = {1.0, spm.x, spm.y};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const double wr = kw.re * ut[a], wi = kw.im * ut[a];
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        are[a][b] = fma(wr, vs[b], are[a][b]);
                        aim[a][b] = fma(wi, vs[b], aim[a][b]);
                    }
                }
            } else {
                // H = w G (ikr - 1) / r^2 and d = x - y; with w_t = J_t (xi, eta), w_s likewise, the four sums
                // PB = sum w_t . (H w_s x d), PC = sum (H d) x w_t, QB = sum H w_s x d, QC = sum H d
                const double df[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
                const double d2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
                const double d = sqrt(d2);
                const cplx f = cmul(kw, cplx{(-ki * d - 1.0) / d2, kr * d / d2});
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
                pbr = fma(f.re, pb, pbr);
                pbi = fma(f.im, pb, pbi);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    pcr[c] = fma(f.re, dxw[c], pcr[c]);
                    pci[c] = fma(f.im, dxw[c], pci[c]);
                    qbr[c] = fma(f.re, wxd[c], qbr[c]);
                    qbi[c] = fma(f.im, wxd[c], qbi[c]);
                    qcr[c] = fma(f.re, df[c], qcr[c]);
                    qci[c] = fma(f.im, df[c], qci[c]);
                }
            }
        }
    }

    // reduce across the warp
    constexpr bool HYP_K = HYP && ASM != BEMPPCUDA_ASM_LAPLACE_HYP;
    constexpr bool MFIE = ASM == BEMPPCUDA_ASM_MFIE;
    if (HYP_K) {
        sre = warp_sum(sre);
        sim = warp_sum(sim);
    }
    if (MFIE) {
        pbr = warp_sum(pbr);
        pbi = warp_sum(pbi);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pcr[c] = warp_sum(pcr[c]);
            pci[c] = warp_sum(pci[c]);
            qbr[c] = warp_sum(qbr[c]);
            qbi[c] = warp_sum(qbi[c]);
            qcr[c] = warp_sum(qcr[c]);
            qci[c] = warp_sum(qci[c]);
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool live = MFIE ? false : (ASM == BEMPPCUDA_ASM_LAPLACE_HYP) ? (i == 0 && j == 0)
                                                                             : (i < nt && j < ns);
            if (live) {
                are[i][j] = warp_sum(are[i][j]);
                aim[i][j] = warp_sum(aim[i][j]);
            }
        }
    if (lane != 0) return;
    const double scale = gt.ie * gs.ie;
    double eb_re[3][3], eb_im[3][3];  // EFIE / MFIE block from the moments or sums (the |J| factors cancel)
    if (MFIE) mfie_block(pbr, pbi, pcr, pci, qbr, qbi, qcr, qci, gt.j0, gt.j1, gs.j0, gs.j1, eb_re, eb_im);
    if (ASM == BEMPPCUDA_ASM_EFIE) {
        if (ki != 0.0)
            efie_block<true>(are, aim, gt.j0, gt.j1, gs.j0, gs.j1, kr, ki, eb_re, eb_im);
        else
            efie_block<false>(are, aim, gt.j0, gt.j1, gs.j0, gs.j1, kr, 0.0, eb_re, eb_im);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        if (i >= nt) continue;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            if (j >= ns) continue;
            double vr, vi;
            if (ASM == BEMPPCUDA_ASM_LAPLACE_HYP) {
                vr = are[0][0] * scale * cp[i][j];
                vi = 0.0;
            } else if (HYP_K) {
                // c = -k^2 (Helmholtz, complex k allowed) or +omega^2 (modified Helmholtz)
                const double k2r = ASM == BEMPPCUDA_ASM_HELM_HYP ? -(kr * kr - ki * ki) : kr * kr;
                const double k2i = ASM == BEMPPCUDA_ASM_HELM_HYP ? -(2.0 * kr * ki) : 0.0;
                const double mr = are[i][j] * normal_prod, mi = aim[i][j] * normal_prod;
                vr = fma(cp[i][j], sre, fma(k2r, mr, -k2i * mi)) * scale;
                vi = fma(cp[i][j], sim, fma(k2r, mi, k2i * mr)) * scale;
            } else if (MAXWELL) {
                const double f = edge_length(prm.g, prm.ne, t, i) * edge_length(prm.g, prm.ne, s, j);
                vr = eb_re[i][j] * f;
                vi = eb_im[i][j] * f;
            } else {
                double f = scale;
                if (MAXWELL) f *= edge_length(prm.g, prm.ne, t, i) * edge_length(prm.g, prm.ne, s, j);
                vr = are[i][j] * f;
                vi = aim[i][j] * f;
            }
            if (prm.values) {
                const int64_t idx = (k * nt + i) * ns + j;
                if (prm.is_complex) {
                    double *o = reinterpret_cast<double *>(prm.values) + 2 * idx;
                    o[0] += vr;
                    o[1] += vi;
                } else {
                    reinterpret_cast<double *>(prm.values)[idx] += vr;
                }
            } else {
                const double mt = prm.tmult[t * nt + i], ms = prm.smult[s * ns + j];
                if (mt == 0.0 || ms == 0.0) continue;
                const int64_t row = prm.tl2g[t * nt + i], col = prm.sl2g[s * ns + j];
                if (t == s && nt == 1 && ns == 1) vr += prm.diag_shift * 0.5 * gt.ie;
                const double m = mt * ms;
                if (prm.is_complex) {
                    double *o = reinterpret_cast<double *>(prm.dense) + 2 * (row * prm.ld + col);
                    atomicAdd(o, vr * m);
                    atomicAdd(o + 1, vi * m);
                } else {
                    atomicAdd(reinterpret_cast<double *>(prm.dense) + row * prm.ld + col, vr * m);
                }
            }
        }
    }
}

// DP0 scalar kernels (singular_dp0.cuh).
template <int K, int PHC>
__global__ void __launch_bounds__(32 * SING_WARPS) singular_dp0(SingParams prm) {
    const int lane = threadIdx.x & 31;
    const int64_t k = (int64_t)blockIdx.x * SING_WARPS + (threadIdx.x >> 5);
    if (k >= prm.npairs || !pair_in_range(prm, k)) return;
    const int64_t t = prm.te[k], s = prm.se[k];
    // a vertex-adjacent pair in dense mode: the reverse pair's points are these points with the roles
    // exchanged, so the pair with t < s gives both entries and the other one nothing
    const bool mirror = !prm.values && prm.mirror_woff > 0 && (int64_t)prm.woff[k] == prm.mirror_woff;
    if (mirror && t > s) return;
    Geom gt, gs;
    load_geom(prm.g, prm.ne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
    load_geom(prm.g, prm.ne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    double vr, vi, ur = 0.0, ui = 0.0;
    if (mirror)
        sing_dp0_pair<K, PHC>(prm.g, prm.ne, t, s, gt, gs, prm.p, reinterpret_cast<const double2 *>(prm.tp),
                              reinterpret_cast<const double2 *>(prm.sp), prm.w, prm.toff[k], prm.soff[k],
                              prm.woff[k], (int)prm.npts[k], &vr, &vi, &ur, &ui);
    else
        sing_dp0_value<K, PHC>(prm.g, prm.ne, t, s, gt, gs, prm.p, reinterpret_cast<const double2 *>(prm.tp),
                               reinterpret_cast<const double2 *>(prm.sp), prm.w, prm.toff[k], prm.soff[k],
                               prm.woff[k], (int)prm.npts[k], &vr, &vi);
    if (lane != 0) return;
    const double scale = BC_INV_4PI * gt.ie * gs.ie;
    vr *= scale;
    vi *= scale;
    if (mirror) {
        // the (s, t) entry
        const double mt = prm.tmult[s], ms = prm.smult[t];
        if (mt != 0.0 && ms != 0.0) {
            const int64_t row = prm.tl2g[s], col = prm.sl2g[t];
            const double mm = mt * ms * scale;
            if (prm.is_complex) {
                double *o = reinterpret_cast<double *>(prm.dense) + 2 * (row * prm.ld + col);
                atomicAdd(o, ur * mm);
                atomicAdd(o + 1, ui * mm);
            } else {
                atomicAdd(reinterpret_cast<double *>(prm.dense) + row * prm.ld + col, ur * mm);
            }
        }
    }
    if (prm.values) {
        if (prm.is_complex) {
            double *o = reinterpret_cast<double *>(prm.values) + 2 * k;
            o[0] += vr;
            o[1] += vi;
        } else {
            reinterpret_cast<double *>(prm.values)[k] += vr;
        }
        return;
    }
    const double mt = prm.tmult[t], ms = prm.smult[s];
    if (mt == 0.0 || ms == 0.0) return;
    const int64_t row = prm.tl2g[t], col = prm.sl2g[s];
    if (t == s) vr += prm.diag_shift * 0.5 * gt.ie;
    const double mm = mt * ms;
    if (prm.is_complex) {
        double *o = reinterpret_cast<double *>(prm.dense) + 2 * (row * prm.ld + col);
        atomicAdd(o, vr * mm);
        atomicAdd(o + 1, vi * mm);
    } else {
        atomicAdd(reinterpret_cast<double *>(prm.dense) + row * prm.ld + col, vr * mm);
    }
}

template <int K>
static cudaError_t launch_sing_dp0(const SingParams &prm, int phase_class, cudaStream_t st) {
    const unsigned blocks = (unsigned)((prm.npairs + SING_WARPS - 1) / SING_WARPS);
    if constexpr (!SingDp0Traits<K>::helm) {  // no phase: one instance
        singular_dp0<K, 0><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    } else {
        if (phase_class == 3)  // complex wavenumber
            singular_dp0<K, 3><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else if (phase_class == 2)
            singular_dp0<K, 2><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else if (phase_class == 1)
            singular_dp0<K, 1><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else
            singular_dp0<K, 0><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    }
    return cudaGetLastError();
}

}  // namespace bc

#include "singular_p1.cuh"   // singular_p1 and singular_rwg, on SingParams, pair_in_range and SING_WARPS above
#include "singular_rwg.cuh"

namespace bc {

template <int ASM, int K>
static cudaError_t launch_sing_p1(const SingParams &prm, int phase_class, cudaStream_t st) {
    const unsigned blocks = (unsigned)((prm.npairs + SING_WARPS - 1) / SING_WARPS);
    if constexpr (!SingDp0Traits<K>::helm) {
        singular_p1<ASM, K, 0><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    } else {
        if (phase_class == 3)
            singular_p1<ASM, K, 3><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else if (phase_class == 2)
            singular_p1<ASM, K, 2><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else if (phase_class == 1)
            singular_p1<ASM, K, 1><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
        else
            singular_p1<ASM, K, 0><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    }
    return cudaGetLastError();
}

template <int ASM>
static cudaError_t launch_sing_rwg(const SingParams &prm, int phase_class, cudaStream_t st) {
    const unsigned blocks = (unsigned)((prm.npairs + SING_WARPS - 1) / SING_WARPS);
    if (phase_class == 3)
        singular_rwg<ASM, 3><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    else if (phase_class == 2)
        singular_rwg<ASM, 2><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    else if (phase_class == 1)
        singular_rwg<ASM, 1><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    else
        singular_rwg<ASM, 0><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    return cudaGetLastError();
}

// Three shapes on both sides: P1 x P1 for the scalar kernels without the combined field and the
// three hypersingular operators, RWG / SNC for the Maxwell operators; false when the pair list needs
// the generic kernel
static bool launch_p1_pairs(const bemppcuda_singular_args *a, const SingParams &prm, int phase_class,
                            cudaStream_t st, cudaError_t *err) {
    if (prm.nt != 3 || prm.ns != 3) return false;
    switch (a->assembly) {
    case BEMPPCUDA_ASM_SCALAR:
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: *err = launch_sing_p1<0, BEMPPCUDA_LAPLACE_SLP>(prm, 0, st); return true;
        case BEMPPCUDA_LAPLACE_DLP: *err = launch_sing_p1<0, BEMPPCUDA_LAPLACE_DLP>(prm, 0, st); return true;
        case BEMPPCUDA_LAPLACE_ADLP: *err = launch_sing_p1<0, BEMPPCUDA_LAPLACE_ADLP>(prm, 0, st); return true;
        case BEMPPCUDA_HELMHOLTZ_SLP:
            *err = launch_sing_p1<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, phase_class, st);
            return true;
        case BEMPPCUDA_HELMHOLTZ_DLP:
            *err = launch_sing_p1<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, phase_class, st);
            return true;
        case BEMPPCUDA_HELMHOLTZ_ADLP:
            *err = launch_sing_p1<0, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, phase_class, st);
            return true;
        case BEMPPCUDA_MODHELM_SLP: *err = launch_sing_p1<0, BEMPPCUDA_MODHELM_SLP>(prm, 0, st); return true;
        case BEMPPCUDA_MODHELM_DLP: *err = launch_sing_p1<0, BEMPPCUDA_MODHELM_DLP>(prm, 0, st); return true;
        case BEMPPCUDA_MODHELM_ADLP: *err = launch_sing_p1<0, BEMPPCUDA_MODHELM_ADLP>(prm, 0, st); return true;
        default: return false;
        }
    case BEMPPCUDA_ASM_LAPLACE_HYP: *err = launch_sing_p1<1, BEMPPCUDA_LAPLACE_SLP>(prm, 0, st); return true;
    case BEMPPCUDA_ASM_HELM_HYP: *err = launch_sing_p1<2, BEMPPCUDA_HELMHOLTZ_SLP>(prm, phase_class, st); return true;
    case BEMPPCUDA_ASM_MODHELM_HYP: *err = launch_sing_p1<3, BEMPPCUDA_MODHELM_SLP>(prm, 0, st); return true;
    case BEMPPCUDA_ASM_EFIE: *err = launch_sing_rwg<BEMPPCUDA_ASM_EFIE>(prm, phase_class, st); return true;
    case BEMPPCUDA_ASM_MFIE: *err = launch_sing_rwg<BEMPPCUDA_ASM_MFIE>(prm, phase_class, st); return true;
    default: return false;
    }
}

template <int ASM, int K>
static cudaError_t launch_sing(const SingParams &prm, cudaStream_t st) {
    const unsigned blocks = (unsigned)((prm.npairs + SING_WARPS - 1) / SING_WARPS);
    singular_pairs<ASM, K><<<blocks, 32 * SING_WARPS, 0, st>>>(prm);
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

int bc_singular_launch(const bemppcuda_singular_args *a, cudaStream_t st) {
    SingParams prm;
    prm.g = a->grid.geom;
    prm.ne = a->grid.nelements;
    prm.te = a->test_elements;
    prm.se = a->trial_elements;
    prm.toff = a->test_offsets;
    prm.soff = a->trial_offsets;
    prm.woff = a->weights_offsets;
    prm.npts = a->npoints;
    prm.tp = a->test_points;
    prm.sp = a->trial_points;
    prm.w = a->weights;
    prm.npairs = a->npairs;
    prm.tnm = a->test.normal_mult;
    prm.snm = a->trial.normal_mult;
    prm.nt = a->test.nshape;
    prm.ns = a->trial.nshape;
    prm.is_complex = a->is_complex;
    prm.pad = 0;
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    prm.values = a->values;
    prm.dense = a->dense;
    prm.ld = a->ld;
    prm.tl2g = a->test.l2g;
    prm.sl2g = a->trial.l2g;
    prm.tmult = a->test.mult;
    prm.smult = a->trial.mult;
    prm.diag_shift = a->diag_shift;
    prm.ntab = a->npoints_table;
    prm.nw = a->nweights;
    prm.mirror_woff = a->mirror_weights_offset;
    if (prm.npairs == 0) return BEMPPCUDA_OK;
    cudaError_t err = cudaSuccess;
    const bool real_k = a->params[1] == 0.0;
    // a complex wavenumber takes phase class 3 (no centroid factoring)
    const double theta = fabs(a->params[0]) * a->phase_radius;
    const int phase_class = !real_k ? 3 : a->phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
    if (launch_p1_pairs(a, prm, phase_class, st, &err)) {
        if (err != cudaSuccess) {
            bc_set_error("singular assembly launch failed: %s", cudaGetErrorString(err));
            return BEMPPCUDA_ERR_CUDA;
        }
        return BEMPPCUDA_OK;
    }
    if (a->assembly == BEMPPCUDA_ASM_SCALAR && prm.nt == 1 && prm.ns == 1 &&
        (a->kernel <= BEMPPCUDA_MODHELM_ADLP || a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED)) {
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: err = launch_sing_dp0<BEMPPCUDA_LAPLACE_SLP>(prm, 0, st); break;
        case BEMPPCUDA_LAPLACE_DLP: err = launch_sing_dp0<BEMPPCUDA_LAPLACE_DLP>(prm, 0, st); break;
        case BEMPPCUDA_LAPLACE_ADLP: err = launch_sing_dp0<BEMPPCUDA_LAPLACE_ADLP>(prm, 0, st); break;
        case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_sing_dp0<BEMPPCUDA_HELMHOLTZ_SLP>(prm, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_sing_dp0<BEMPPCUDA_HELMHOLTZ_DLP>(prm, phase_class, st); break;
        case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_sing_dp0<BEMPPCUDA_HELMHOLTZ_ADLP>(prm, phase_class, st); break;
        case BEMPPCUDA_MODHELM_SLP: err = launch_sing_dp0<BEMPPCUDA_MODHELM_SLP>(prm, 0, st); break;
        case BEMPPCUDA_MODHELM_DLP: err = launch_sing_dp0<BEMPPCUDA_MODHELM_DLP>(prm, 0, st); break;
        case BEMPPCUDA_MODHELM_ADLP: err = launch_sing_dp0<BEMPPCUDA_MODHELM_ADLP>(prm, 0, st); break;
        default: err = launch_sing_dp0<BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, phase_class, st); break;
        }
        if (err != cudaSuccess) {
            bc_set_error("singular assembly launch failed: %s", cudaGetErrorString(err));
            return BEMPPCUDA_ERR_CUDA;
        }
        return BEMPPCUDA_OK;
    }
    switch (a->assembly) {
    case BEMPPCUDA_ASM_SCALAR:
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: err = launch_sing<0, BEMPPCUDA_LAPLACE_SLP>(prm, st); break;
        case BEMPPCUDA_LAPLACE_DLP: err = launch_sing<0, BEMPPCUDA_LAPLACE_DLP>(prm, st); break;
        case BEMPPCUDA_LAPLACE_ADLP: err = launch_sing<0, BEMPPCUDA_LAPLACE_ADLP>(prm, st); break;
        case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_sing<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
        case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_sing<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, st); break;
        case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_sing<0, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, st); break;
        case BEMPPCUDA_MODHELM_SLP: err = launch_sing<0, BEMPPCUDA_MODHELM_SLP>(prm, st); break;
        case BEMPPCUDA_MODHELM_DLP: err = launch_sing<0, BEMPPCUDA_MODHELM_DLP>(prm, st); break;
        case BEMPPCUDA_MODHELM_ADLP: err = launch_sing<0, BEMPPCUDA_MODHELM_ADLP>(prm, st); break;
        case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_sing<0, BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, st); break;
        default: bc_set_error("kernel %d not valid for singular assembly", a->kernel); return BEMPPCUDA_ERR_INVALID;
        }
        break;
    case BEMPPCUDA_ASM_LAPLACE_HYP: err = launch_sing<1, BEMPPCUDA_LAPLACE_SLP>(prm, st); break;
    case BEMPPCUDA_ASM_HELM_HYP: err = launch_sing<2, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
    case BEMPPCUDA_ASM_MODHELM_HYP: err = launch_sing<3, BEMPPCUDA_MODHELM_SLP>(prm, st); break;
    case BEMPPCUDA_ASM_EFIE: err = launch_sing<4, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
    case BEMPPCUDA_ASM_MFIE: err = launch_sing<5, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
    default: bc_set_error("assembly type %d unknown", a->assembly); return BEMPPCUDA_ERR_INVALID;
    }
    if (err != cudaSuccess) {
        bc_set_error("singular assembly launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
