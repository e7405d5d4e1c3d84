// Regular (non-adjacent) element-pair quadrature for dense Galerkin assembly.
//
// Replaces the regular assemblers of bempp_cl/core/numba_kernels.py:
// default_scalar_regular_kernel (:980-1074), laplace/helmholtz/modified
// hypersingular_regular (:1078-1467), maxwell_efield_regular_assembler
// (:1853-1970) and maxwell_mfield_regular_assembler (:2151-2278).
//
// Two kernels:
//  * regular_dp0<K, MIXED>: piecewise-constant test and trial spaces with the
//    identity dof map, 6-point rule.  One thread owns one trial element
//    (a matrix column) and sweeps a block of test elements (rows) staged in
//    shared memory; the 6 trial quadrature points stay in registers; every
//    matrix entry is written exactly once (coalesced along the row).
//    MIXED evaluates the 36 quadrature-point pairs in FP32 relative to the
//    element centroids: the centroid distance r_c and exp(i k r_c) are FP64,
//    per point only the offset r - r_c = (2 D.e + e.e) / (r + r_c) enters
//    the FP32 phase, so the phase error stays ~1e-7 rad independently of
//    k r.  The 6-point inner sums are FP32, the per-entry sum is FP64.
//  * regular_p1<ASM, K, ...> (p1.cuh): scalar and hypersingular operators on
//    P1 / DP1 / P0 spaces, 6-point rule, real wavenumber.
//  * regular_rwg<ASM, ...> (rwg.cuh): Maxwell electric / magnetic field on
//    RWG / SNC spaces, 6-point rule, real nonzero wavenumber.
//  * regular_generic<ASM, K>: every other scalar / hypersingular / Maxwell
//    assembly with 1 or 3 shape functions and any rule (<= 16 points).  One
//    thread per element pair; the local nshape x nshape block is scattered
//    with atomicAdd into the (pre-zeroed or accumulating) result.
#include <cstdio>

#include "dp0_sym.cuh"
#include "p1.cuh"
#include "p1_mixed.cuh"
#include "rwg.cuh"

namespace bc {

// --------------------------------------------------------------------------------------------
// Generic element-pair kernel
// --------------------------------------------------------------------------------------------
constexpr int GEN_THREADS = 128;
constexpr int GEN_TCHUNK = 16;

__device__ __forceinline__ void atomic_add_out(void *result, int is_complex, int64_t ld, int64_t row, int64_t col,
                                               double re, double im) {
    if (is_complex) {
        double *o = reinterpret_cast<double *>(result) + 2 * (row * ld + col);
        atomicAdd(o, re);
        atomicAdd(o + 1, im);
    } else {
        atomicAdd(reinterpret_cast<double *>(result) + row * ld + col, re);
    }
}

template <int ASM, int K>
__global__ void __launch_bounds__(GEN_THREADS) regular_generic(RegParams prm, QuadRule rule) {
    __shared__ double s_x[GEN_TCHUNK][BEMPPCUDA_MAX_REGULAR_POINTS][3];
    __shared__ double s_n[GEN_TCHUNK][3];
    __shared__ double s_ie[GEN_TCHUNK];
    __shared__ int s_v[GEN_TCHUNK][3];

    const int nq = rule.nq;
    const int64_t t0 = (int64_t)blockIdx.y * GEN_TCHUNK;
    const int tcount = (int)min((int64_t)GEN_TCHUNK, prm.ntest - t0);
    for (int idx = threadIdx.x; idx < tcount; idx += blockDim.x) {
        const int64_t t = prm.tsup[t0 + idx];
        Geom g;
        load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, g);
        for (int p = 0; p < nq; ++p) {
            double x[3];
            to_global(g, rule.x[p], rule.y[p], x);
#pragma unroll
            for (int d = 0; d < 3; ++d) s_x[idx][p][d] = x[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s_n[idx][d] = g.n[d];
            s_v[idx][d] = __ldg(prm.tel + 3 * t + d);
        }
        s_ie[idx] = g.ie;
    }
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * GEN_THREADS + threadIdx.x;
    if (si >= prm.ntrial) return;
    const int64_t s = prm.ssup[si];
    Geom gs;
    load_geom(prm.sg, prm.sne, s, prm.snm ? (double)prm.snm[s] : 1.0, gs);
    const int sv0 = __ldg(prm.sel + 3 * s), sv1 = __ldg(prm.sel + 3 * s + 1), sv2 = __ldg(prm.sel + 3 * s + 2);
    const int nt = prm.tnshape, ns = prm.snshape;
    const double kr = prm.p[0], ki = prm.p[1];
    constexpr bool HYP = (ASM == BEMPPCUDA_ASM_LAPLACE_HYP || ASM == BEMPPCUDA_ASM_HELM_HYP ||
                          ASM == BEMPPCUDA_ASM_MODHELM_HYP);
    constexpr bool MAXWELL = (ASM == BEMPPCUDA_ASM_EFIE || ASM == BEMPPCUDA_ASM_MFIE);
    double curl_s[3][3];
    if (HYP) surface_curls(prm.sg, prm.sne, s, gs.n, curl_s);
    double el_s[3] = {1.0, 1.0, 1.0};
    if (MAXWELL)
        for (int j = 0; j < 3; ++j) el_s[j] = edge_length(prm.sg, prm.sne, s, j);

    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t t = prm.tsup[t0 + tt];
        if (prm.grids_identical) {
            const int a0 = s_v[tt][0], a1 = s_v[tt][1], a2 = s_v[tt][2];
            if ((a0 == sv0) | (a0 == sv1) | (a0 == sv2) | (a1 == sv0) | (a1 == sv1) | (a1 == sv2) | (a2 == sv0) |
                (a2 == sv1) | (a2 == sv2))
                continue;
        }
        const double tn[3] = {s_n[tt][0], s_n[tt][1], s_n[tt][2]};
        double lre[3][3], lim[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) lre[i][j] = lim[i][j] = 0.0;

        Geom gt;  // test geometry for the Piola transform / curls
        double curl_t[3][3];
        if (HYP || MAXWELL) {
            load_geom(prm.tg, prm.tne, t, prm.tnm ? (double)prm.tnm[t] : 1.0, gt);
            if (HYP) surface_curls(prm.tg, prm.tne, t, gt.n, curl_t);
        }
        const double normal_prod = tn[0] * gs.n[0] + tn[1] * gs.n[1] + tn[2] * gs.n[2];
        double cp[3][3];
        if (HYP) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    cp[i][j] = curl_t[i][0] * curl_s[j][0] + curl_t[i][1] * curl_s[j][1] + curl_t[i][2] * curl_s[j][2];
        }
        for (int p = 0; p < nq; ++p) {
            const double xp[3] = {s_x[tt][p][0], s_x[tt][p][1], s_x[tt][p][2]};
            double phi_t[3];
            scalar_shape(nt, rule.x[p], rule.y[p], phi_t);
            double bt[3][3];
            if (MAXWELL) rwg_values(gt, rule.x[p], rule.y[p], bt);
            for (int q = 0; q < nq; ++q) {
                double yq[3];
                to_global(gs, rule.x[q], rule.y[q], yq);
                const cplx kv = greens<K>(xp, yq, tn, gs.n, prm.p);
                const double wf = rule.w[p] * rule.w[q];
                const cplx tmp = cscale(kv, wf);
                double phi_s[3];
                scalar_shape(ns, rule.x[q], rule.y[q], phi_s);
                if (ASM == BEMPPCUDA_ASM_SCALAR) {
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            if (i < nt && j < ns) {
                                const double f = phi_t[i] * phi_s[j];
                                lre[i][j] = fma(tmp.re, f, lre[i][j]);
                                lim[i][j] = fma(tmp.im, f, lim[i][j]);
                            }
                        }
                } else if (HYP) {
                    // curl.curl - k^2 phi psi n.n (Helmholtz), + k^2 (modified), curl.curl (Laplace)
                    double k2r = 0.0, k2i = 0.0;
                    if (ASM == BEMPPCUDA_ASM_HELM_HYP) {
                        k2r = -(kr * kr - ki * ki);
                        k2i = -(2.0 * kr * ki);
                    } else if (ASM == BEMPPCUDA_ASM_MODHELM_HYP) {
                        k2r = kr * kr;
                    }
#pragma unroll
                    for (int i = 0; i < 3; ++i)
#pragma unroll
                        for (int j = 0; j < 3; ++j) {
                            const double m = phi_t[i] * phi_s[j] * normal_prod;
                            const cplx fac = {cp[i][j] + k2r * m, k2i * m};
                            const cplx v = cmul(tmp, fac);
                            lre[i][j] += v.re;
                            lim[i][j] += v.im;
                        }
                } else {
                    double bs[3][3];
                    rwg_values(gs, rule.x[q], rule.y[q], bs);
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
                        // -i k b_t.b_s - 4 / (i k |J_t| |J_s|)
                        const double div = 4.0 / (gt.ie * gs.ie);
                        // 1 / (i k) = -i conj(k) / |k|^2
                        const double kk = kr * kr + ki * ki;
                        const cplx inv_ik = {-ki / kk, -kr / kk};
                        const cplx mik = {ki, -kr};  // -i k
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) {
                                const double dot = bt[i][0] * bs[j][0] + bt[i][1] * bs[j][1] + bt[i][2] * bs[j][2];
                                const cplx fac = {mik.re * dot - div * inv_ik.re, mik.im * dot - div * inv_ik.im};
                                const cplx v = cmul(tmp, fac);
                                lre[i][j] += v.re;
                                lim[i][j] += v.im;
                            }
                    } else {
                        const double df[3] = {xp[0] - yq[0], xp[1] - yq[1], xp[2] - yq[2]};
                        const double dist2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
                        const double dist = sqrt(dist2);
                        // (i k dist - 1) / dist^2
                        const cplx f = {(-ki * dist - 1.0) / dist2, kr * dist / dist2};
                        const cplx tf = cmul(tmp, f);
#pragma unroll
                        for (int i = 0; i < 3; ++i)
#pragma unroll
                            for (int j = 0; j < 3; ++j) {
                                const double c0 = bt[i][1] * bs[j][2] - bt[i][2] * bs[j][1];
                                const double c1 = bt[i][2] * bs[j][0] - bt[i][0] * bs[j][2];
                                const double c2 = bt[i][0] * bs[j][1] - bt[i][1] * bs[j][0];
                                const double tr = df[0] * c0 + df[1] * c1 + df[2] * c2;
                                lre[i][j] += tf.re * tr;
                                lim[i][j] += tf.im * tr;
                            }
                    }
                }
            }
        }
        const double scale = s_ie[tt] * gs.ie;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (i >= nt) continue;
            const double mt = prm.tmult[t * nt + i];
            if (mt == 0.0) continue;
            const int64_t row = prm.tl2g[t * nt + i];
            const double elt = MAXWELL ? edge_length(prm.tg, prm.tne, t, i) : 1.0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                if (j >= ns) continue;
                const double ms = prm.smult[s * ns + j];
                if (ms == 0.0) continue;
                const int64_t col = prm.sl2g[s * ns + j];
                const double f = scale * mt * ms * elt * el_s[j];
                atomic_add_out(prm.result, prm.is_complex, prm.ld, row, col, lre[i][j] * f, lim[i][j] * f);
            }
        }
    }
}

// Symmetric sweeps: blockIdx.x = column block, blockIdx.y = row chunk; chunks
// that start below the block's last column have no pair i <= j and exit
// before touching shared memory.
template <int K, int PHC, bool STRIPE = false>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_fp64_sym(RegParams prm, QuadRule rule, int64_t row0,
                                                                    int64_t row1, int tile_rows) {
    const int64_t t0 = row0 + (int64_t)blockIdx.y * tile_rows;
    if (t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;
    __shared__ TestBlock64s sb;
    regular_dp0_fp64_sym_tile<K, PHC, STRIPE>(prm, rule, blockIdx.x, t0, (int)min((int64_t)tile_rows, row1 - t0),
                                              sb);
}

// CTAs per SM the mixed symmetric sweep is compiled for (register cap 170 at
// 3): timed at L6, 3 and 4 are equal, 2 is 10 % slower.
#ifndef BC_MSYM_MIN_BLOCKS
#define BC_MSYM_MIN_BLOCKS 3
#endif

template <int K, int PHC, bool STRIPE = false, bool CK = false>
__global__ void __launch_bounds__(DP0_THREADS, BC_MSYM_MIN_BLOCKS) regular_dp0_mixed_sym(RegParams prm, QuadRule rule,
                                                                                      int64_t row0, int64_t row1,
                                                                                      int tile_rows) {
    const int64_t t0 = row0 + (int64_t)blockIdx.y * tile_rows;
    if (t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;
    __shared__ TestBlock32q sb;
    regular_dp0_mixed_sym_tile<K, PHC, STRIPE, CK>(prm, rule, blockIdx.x, t0,
                                                   (int)min((int64_t)tile_rows, row1 - t0), sb);
}

// The mixed symmetric sweep in its phase class, real or (Helmholtz) complex wavenumber.
template <int K, bool STRIPE, bool CK>
static void mixed_sym_phase(const RegParams &prm, const QuadRule &rule, int phase_class, int64_t row0, int64_t row1,
                            int tile_rows, dim3 sgrid, cudaStream_t st) {
    if (phase_class == 2)
        regular_dp0_mixed_sym<K, 2, STRIPE, CK><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
    else if (phase_class == 1)
        regular_dp0_mixed_sym<K, 1, STRIPE, CK><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
    else
        regular_dp0_mixed_sym<K, 0, STRIPE, CK><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
}

template <int K, bool STRIPE>
static void launch_mixed_sym(const RegParams &prm, const QuadRule &rule, int phase_class, int64_t row0, int64_t row1,
                             int tile_rows, dim3 sgrid, cudaStream_t st) {
    if constexpr (KernelTraits<K>::helm) {
        if (prm.p[1] != 0.0) {
            mixed_sym_phase<K, STRIPE, true>(prm, rule, phase_class, row0, row1, tile_rows, sgrid, st);
            return;
        }
    }
    mixed_sym_phase<K, STRIPE, false>(prm, rule, phase_class, row0, row1, tile_rows, sgrid, st);
}

// Kernels with a stripe-mode instance (the multi-GPU symmetric stripes): the Helmholtz family, the
// combined field and the Laplace single layer.
template <int K>
constexpr bool stripe_kernel() {
    return K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP ||
           K == BEMPPCUDA_HELMHOLTZ_COMBINED || K == BEMPPCUDA_LAPLACE_SLP;
}

// The symmetric sweep of launch_dp0 in stripe mode (real or complex wavenumber; mixed or FP64).
template <int K>
static cudaError_t launch_dp0_stripe(const RegParams &prm, const QuadRule &rule, int mixed, int phase_class,
                                     int64_t row0, int64_t row1, int tile_rows, dim3 sgrid, cudaStream_t st) {
    if constexpr (stripe_kernel<K>()) {
        if (mixed) {
            launch_mixed_sym<K, true>(prm, rule, phase_class, row0, row1, tile_rows, sgrid, st);
        } else if (!KernelTraits<K>::helm) {
            regular_dp0_fp64_sym<K, 0, true><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
        } else if (prm.p[1] != 0.0) {
            regular_dp0_fp64_sym<K, 3, true><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
        } else if (phase_class == 2) {
            regular_dp0_fp64_sym<K, 2, true><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
        } else if (phase_class == 1) {
            regular_dp0_fp64_sym<K, 1, true><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
        } else {
            regular_dp0_fp64_sym<K, 0, true><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
        }
        return cudaGetLastError();
    } else {
        return cudaErrorInvalidValue;
    }
}

template <int K>
static cudaError_t launch_dp0(const RegParams &prm, const QuadRule &rule, int mixed, int phase_class, bool sym,
                              int64_t row0, int64_t row1, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS), (unsigned)((prm.ntest + DP0_TCHUNK - 1) / DP0_TCHUNK));
    if constexpr (SymTraits<K>::supported) {
        // same DP0 space on both sides; the mixed tiles need Re k > 0 or omega > 0 (scaled units; a
        // complex k adds the amplitude split), the FP64 tiles take a complex k as phase class 3
        const bool helm = KernelTraits<K>::helm;
        const bool ck_sym = helm && prm.p[1] != 0.0;
        const bool sweep_ok = helm || KernelTraits<K>::modhelm ? (!mixed || prm.p[0] > 0.0) : true;
        if (sym && sweep_ok) {
            // rows per tile: 32, or 16 / 8 when 32-row tiles would leave the GPU under four waves of
            // working CTAs (about half the tiles lie below the diagonal and exit; 3 CTAs per SM)
            int tile_rows = DP0_TCHUNK;
            const int64_t wave = (int64_t)bc_sm_count() * 3;
            while (tile_rows > 8 && (int64_t)grid.x * ((row1 - row0 + tile_rows - 1) / tile_rows) / 2 < 4 * wave)
                tile_rows /= 2;
            const dim3 sgrid(grid.x, (unsigned)((row1 - row0 + tile_rows - 1) / tile_rows));
            if (prm.tresult) return launch_dp0_stripe<K>(prm, rule, mixed, phase_class, row0, row1, tile_rows, sgrid, st);
            if (mixed) {
                launch_mixed_sym<K, false>(prm, rule, phase_class, row0, row1, tile_rows, sgrid, st);
                return cudaGetLastError();
            }
            if constexpr (!KernelTraits<K>::helm) {  // no phase: one instance
                regular_dp0_fp64_sym<K, 0><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
            } else {
                if (ck_sym)
                    regular_dp0_fp64_sym<K, 3><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
                else if (phase_class == 2)
                    regular_dp0_fp64_sym<K, 2><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
                else if (phase_class == 1)
                    regular_dp0_fp64_sym<K, 1><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
                else
                    regular_dp0_fp64_sym<K, 0><<<sgrid, DP0_THREADS, 0, st>>>(prm, rule, row0, row1, tile_rows);
            }
            return cudaGetLastError();
        }
    }
    const bool ck = prm.p[1] != 0.0 && KernelTraits<K>::helm;
    // the packed path measures lengths in units of 1/k: Helmholtz needs k > 0
    const bool packed = !KernelTraits<K>::helm || prm.p[0] > 0.0;
    if constexpr (!KernelTraits<K>::modhelm) {
        if (mixed && !ck && packed) {
            if (phase_class == 2)
                regular_dp0_mixed2<K, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            else if (phase_class == 1)
                regular_dp0_mixed2<K, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            else
                regular_dp0_mixed2<K, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            return cudaGetLastError();
        }
    }
    if (row0 != 0 || row1 != prm.ntest) return cudaErrorInvalidValue;  // a row range needs the symmetric sweep
    if (mixed) {
        if (ck)
            regular_dp0_mixed<K, true, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_dp0_mixed<K, false, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_dp0_mixed<K, false, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_dp0_mixed<K, false, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    } else {
        if (ck)
            regular_dp0_fp64<K, true, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_dp0_fp64<K, false, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_dp0_fp64<K, false, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_dp0_fp64<K, false, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    }
    return cudaGetLastError();
}

// Row blocks of the Maxwell sweeps (regular_rwg, regular_p1_mixed on RWG): 32 test elements per
// CTA, or 16 when 32 would leave the GPU under four waves of working CTAs (a symmetric sweep's CTAs
// below the diagonal exit at once; 3 CTAs per SM).  The kernels take their chunk height as
// ceil(ntest / gridDim.y).  L4 (2048 elements), regular pass: electric field 0.52 -> 0.40 ms FP64,
// 0.39 -> 0.31 ms mixed; magnetic field 0.38 -> 0.35 ms mixed.  The P1 scalar kernels keep 32 rows
// as a compile-time height: a runtime one made the mixed hypersingular operator 4 % slower at L5.
static unsigned lin_row_blocks(int64_t ntrial, int64_t ntest, bool sym) {
    static_assert(P1_TCHUNK == 32 && RWG_TCHUNK == 32, "row blocks of 32 or 16 test elements");
    const int64_t cols = (ntrial + DP0_THREADS - 1) / DP0_THREADS;
    const int64_t wave = (int64_t)bc_sm_count() * 3;
    const int rows = cols * ((ntest + 31) / 32) / (sym ? 2 : 1) < 4 * wave ? 16 : 32;
    return (unsigned)((ntest + rows - 1) / rows);
}

template <int ASM, int K, int NT, int NS, bool SYM>
static void launch_p1_phase(const RegParams &prm, const QuadRule &rule, int phase_class, dim3 grid, cudaStream_t st) {
    // the phase classes only concern exp(ikr): one instance for Laplace and modified Helmholtz
    if constexpr (K != BEMPPCUDA_HELMHOLTZ_SLP && K != BEMPPCUDA_HELMHOLTZ_DLP && K != BEMPPCUDA_HELMHOLTZ_ADLP) {
        regular_p1<ASM, K, NT, NS, 0, SYM><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    } else {
        if (phase_class == 3)  // complex wavenumber
            regular_p1<ASM, K, NT, NS, 3, SYM><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_p1<ASM, K, NT, NS, 2, SYM><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_p1<ASM, K, NT, NS, 1, SYM><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_p1<ASM, K, NT, NS, 0, SYM><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    }
}

template <int ASM, int K, int NT, int NS>
static void launch_p1_shapes(const RegParams &prm, const QuadRule &rule, int phase_class, bool sym, dim3 grid,
                             cudaStream_t st) {
    // single layer and hypersingular: symmetric; double / adjoint double layer: each pair
    // also gives the transposed pair's block from the other normal (p1.cuh)
    constexpr bool SYMMETRIC_OP = NT == NS;
    if constexpr (SYMMETRIC_OP) {
        if (sym) {
            launch_p1_phase<ASM, K, NT, NS, true>(prm, rule, phase_class, grid, st);
            return;
        }
    }
    launch_p1_phase<ASM, K, NT, NS, false>(prm, rule, phase_class, grid, st);
}

// Scalar and hypersingular operators on P1 / DP1 / P0 spaces with the 6-point
// rule (p1.cuh).
template <int ASM, int K>
static cudaError_t launch_p1(const RegParams &prm, const QuadRule &rule, int phase_class, bool sym, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS),
              (unsigned)((prm.ntest + P1_TCHUNK - 1) / P1_TCHUNK));
    const int nt = prm.tnshape, ns = prm.snshape;
    if (nt == 3 && ns == 3)
        launch_p1_shapes<ASM, K, 3, 3>(prm, rule, phase_class, sym, grid, st);
    else if (nt == 3)
        launch_p1_shapes<ASM, K, 3, 1>(prm, rule, phase_class, false, grid, st);
    else if (ns == 3)
        launch_p1_shapes<ASM, K, 1, 3>(prm, rule, phase_class, false, grid, st);
    else
        launch_p1_shapes<ASM, K, 1, 1>(prm, rule, phase_class, sym, grid, st);
    return cudaGetLastError();
}

// A <- A + A^T for an n x n matrix with row stride ld, in 32 x 32 tiles: the
// block of tile pair (bi, bj), bi <= bj, reads both tiles and writes both sums.
__device__ __forceinline__ double add_pair(double a, double b) { return a + b; }
__device__ __forceinline__ double2 add_pair(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

template <typename T>
__global__ void __launch_bounds__(256) add_transpose(T *a, int64_t n, int64_t ld) {
    const int64_t bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    __shared__ T s1[32][33], s2[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t r0 = bi * 32, c0 = bj * 32;
    for (int k = ty; k < 32; k += 8) {
        if (r0 + k < n && c0 + tx < n) s1[k][tx] = a[(r0 + k) * ld + c0 + tx];  // tile (bi, bj)
        if (c0 + k < n && r0 + tx < n) s2[k][tx] = a[(c0 + k) * ld + r0 + tx];  // tile (bj, bi)
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        if (r0 + k < n && c0 + tx < n) a[(r0 + k) * ld + c0 + tx] = add_pair(s1[k][tx], s2[tx][k]);
        if (bi != bj && c0 + k < n && r0 + tx < n) a[(c0 + k) * ld + r0 + tx] = add_pair(s2[k][tx], s1[tx][k]);
    }
}

static cudaError_t launch_add_transpose(void *a, int64_t n, int64_t ld, bool is_complex, cudaStream_t st) {
    const int64_t tiles = (n + 31) / 32;
    if (tiles == 0) return cudaSuccess;
    const dim3 grid((unsigned)tiles, (unsigned)tiles), block(32, 8);
    if (is_complex)
        add_transpose<double2><<<grid, block, 0, st>>>(reinterpret_cast<double2 *>(a), n, ld);
    else
        add_transpose<double><<<grid, block, 0, st>>>(reinterpret_cast<double *>(a), n, ld);
    return cudaGetLastError();
}

// Mixed-precision single layer, double layers and hypersingular on P1 spaces (p1_mixed.cuh): Helmholtz
// (phase classes, real or complex k), Laplace and modified Helmholtz (no phase classes).
template <int ASM, int K, bool SYM, bool CK>
static void p1_mixed_phase(const RegParams &prm, const QuadRule &rule, int phase_class, dim3 grid, cudaStream_t st) {
    if constexpr (K != BEMPPCUDA_HELMHOLTZ_SLP && K != BEMPPCUDA_HELMHOLTZ_DLP && K != BEMPPCUDA_HELMHOLTZ_ADLP) {
        regular_p1_mixed<ASM, K, 0, SYM, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    } else {
        if (phase_class == 2)
            regular_p1_mixed<ASM, K, 2, SYM, CK><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_p1_mixed<ASM, K, 1, SYM, CK><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_p1_mixed<ASM, K, 0, SYM, CK><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    }
}

// A P0 space beside a P1 one (scalar operators): per-pair sweep, the general phase class.
template <int K, int NT, int NS>
static void p1_mixed_pair(const RegParams &prm, const QuadRule &rule, dim3 grid, cudaStream_t st) {
    constexpr bool helm = K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP || K == BEMPPCUDA_HELMHOLTZ_ADLP;
    if constexpr (helm) {
        if (prm.p[1] != 0.0) {
            regular_p1_mixed<BEMPPCUDA_ASM_SCALAR, K, 0, false, true, NT, NS><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
            return;
        }
    }
    regular_p1_mixed<BEMPPCUDA_ASM_SCALAR, K, 0, false, false, NT, NS><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
}

template <int ASM, int K>
static cudaError_t launch_p1_mixed(const RegParams &prm, const QuadRule &rule, int phase_class, bool sym,
                                   cudaStream_t st) {
    constexpr bool rwg = ASM == BEMPPCUDA_ASM_EFIE || ASM == BEMPPCUDA_ASM_MFIE;
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS),
              rwg ? lin_row_blocks(prm.ntrial, prm.ntest, sym)
                  : (unsigned)((prm.ntest + P1_TCHUNK - 1) / P1_TCHUNK));
    if constexpr (ASM == BEMPPCUDA_ASM_SCALAR) {
        if (prm.tnshape == 3 && prm.snshape == 1) {
            p1_mixed_pair<K, 3, 1>(prm, rule, grid, st);
            return cudaGetLastError();
        }
        if (prm.tnshape == 1 && prm.snshape == 3) {
            p1_mixed_pair<K, 1, 3>(prm, rule, grid, st);
            return cudaGetLastError();
        }
    }
    constexpr bool helm = K == BEMPPCUDA_HELMHOLTZ_SLP || K == BEMPPCUDA_HELMHOLTZ_DLP ||
                          K == BEMPPCUDA_HELMHOLTZ_ADLP;
    const bool ck = helm && prm.p[1] != 0.0;
    if (ck) {
        if constexpr (helm) {
            if (sym)
                p1_mixed_phase<ASM, K, true, true>(prm, rule, phase_class, grid, st);
            else
                p1_mixed_phase<ASM, K, false, true>(prm, rule, phase_class, grid, st);
        }
    } else if (sym) {
        p1_mixed_phase<ASM, K, true, false>(prm, rule, phase_class, grid, st);
    } else {
        p1_mixed_phase<ASM, K, false, false>(prm, rule, phase_class, grid, st);
    }
    return cudaGetLastError();
}

// Maxwell electric / magnetic field on RWG / SNC spaces, 6-point rule, real
// nonzero wavenumber (rwg.cuh).
template <int ASM>
static cudaError_t launch_rwg(const RegParams &prm, const QuadRule &rule, int phase_class, bool sym, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS), lin_row_blocks(prm.ntrial, prm.ntest, sym));
    if (sym) {
        if (phase_class == 3)  // complex wavenumber
            regular_rwg<ASM, 3, true><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_rwg<ASM, 2, true><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_rwg<ASM, 1, true><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_rwg<ASM, 0, true><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    } else {
        if (phase_class == 3)
            regular_rwg<ASM, 3, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 2)
            regular_rwg<ASM, 2, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else if (phase_class == 1)
            regular_rwg<ASM, 1, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
        else
            regular_rwg<ASM, 0, false><<<grid, DP0_THREADS, 0, st>>>(prm, rule);
    }
    return cudaGetLastError();
}

template <int ASM, int K>
static cudaError_t launch_generic(const RegParams &prm, const QuadRule &rule, cudaStream_t st) {
    dim3 grid((unsigned)((prm.ntrial + GEN_THREADS - 1) / GEN_THREADS), (unsigned)((prm.ntest + GEN_TCHUNK - 1) / GEN_TCHUNK));
    regular_generic<ASM, K><<<grid, GEN_THREADS, 0, st>>>(prm, rule);
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

// Host entry: validated arguments in, kernel launches out.  Returns a status.
int bc_regular_launch(const bemppcuda_regular_args *a, cudaStream_t st) {
    RegParams prm;
    prm.tg = a->test_grid.geom;
    prm.sg = a->trial_grid.geom;
    prm.tne = a->test_grid.nelements;
    prm.sne = a->trial_grid.nelements;
    prm.tel = a->test_grid.elements;
    prm.sel = a->trial_grid.elements;
    prm.tsup = a->test.support;
    prm.ssup = a->trial.support;
    prm.ntest = a->test.nsupport;
    prm.ntrial = a->trial.nsupport;
    prm.tl2g = a->test.l2g;
    prm.sl2g = a->trial.l2g;
    prm.tmult = a->test.mult;
    prm.smult = a->trial.mult;
    prm.tnm = a->test.normal_mult;
    prm.snm = a->trial.normal_mult;
    prm.tnshape = a->test.nshape;
    prm.snshape = a->trial.nshape;
    prm.grids_identical = a->grids_identical;
    prm.is_complex = a->is_complex;
    prm.overwrite = a->overwrite;
    prm.defer_transpose = 0;
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    prm.result = a->result;
    prm.ld = a->ld;
    // R_test + R_trial bounds the centroid distance of two elements that share a vertex
    prm.near_r = a->phase_radius > 0.0 ? a->phase_radius : 0.0;
    prm.tresult = nullptr;
    prm.row0 = prm.col0 = 0;
    if (prm.ntest == 0 || prm.ntrial == 0) return BEMPPCUDA_OK;

    QuadRule rule;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);

    const bool dp0 = a->assembly == BEMPPCUDA_ASM_SCALAR && a->test.nshape == 1 && a->trial.nshape == 1 &&
                     a->test.dof_is_position && a->trial.dof_is_position && a->nq == NQ6 &&
                     (a->kernel <= BEMPPCUDA_MODHELM_ADLP || a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED);
    if (a->overwrite && !dp0) {
        bc_set_error("overwrite mode needs the DP0 fast path (DP0 spaces, identity dofs, 6-point rule)");
        return BEMPPCUDA_ERR_INVALID;
    }
    // mixed precision: DP0 scalar kernels, and the single / double / adjoint double layer and
    // hypersingular operators on P1 spaces (6-point rule): Helmholtz with Re k > 0 (complex result),
    // Laplace and modified Helmholtz with w > 0 (real result)
    const bool helm_k = a->kernel == BEMPPCUDA_HELMHOLTZ_SLP || a->kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
                        a->kernel == BEMPPCUDA_HELMHOLTZ_ADLP;
    const bool lap_k = a->kernel <= BEMPPCUDA_LAPLACE_ADLP;
    const bool mh_k = a->kernel >= BEMPPCUDA_MODHELM_SLP && a->kernel <= BEMPPCUDA_MODHELM_ADLP;
    const bool p1_family =
        (a->assembly == BEMPPCUDA_ASM_SCALAR && (helm_k || lap_k || mh_k)) ||
        (a->assembly == BEMPPCUDA_ASM_HELM_HYP && a->kernel == BEMPPCUDA_HELMHOLTZ_SLP) ||
        (a->assembly == BEMPPCUDA_ASM_LAPLACE_HYP && a->kernel == BEMPPCUDA_LAPLACE_SLP) ||
        (a->assembly == BEMPPCUDA_ASM_MODHELM_HYP && a->kernel == BEMPPCUDA_MODHELM_SLP);
    const bool p1_params = (helm_k && a->params[0] > 0.0 && a->is_complex) ||
                           (lap_k && !a->is_complex) || (mh_k && a->params[0] > 0.0 && !a->is_complex);
    // both sides P1 / DP1, or a P0 space beside a P1 one (scalar operators)
    const bool p1_both = a->test.nshape == 3 && a->trial.nshape == 3 && a->test.shapeset == BEMPPCUDA_SHAPE_P1 &&
                         a->trial.shapeset == BEMPPCUDA_SHAPE_P1;
    const bool p1_p0 = a->assembly == BEMPPCUDA_ASM_SCALAR &&
                       ((a->test.nshape == 3 && a->test.shapeset == BEMPPCUDA_SHAPE_P1 && a->trial.nshape == 1 &&
                         a->trial.shapeset == BEMPPCUDA_SHAPE_P0) ||
                        (a->test.nshape == 1 && a->test.shapeset == BEMPPCUDA_SHAPE_P0 && a->trial.nshape == 3 &&
                         a->trial.shapeset == BEMPPCUDA_SHAPE_P1));
    const bool p1_mixed = a->nq == NQ6 && !a->overwrite && (p1_both || p1_p0) && p1_family && p1_params;
    // ... and the Maxwell electric and magnetic fields on RWG / SNC (same FP32 core; 6-point rule,
    // Re k > 0)
    const bool rwg_mixed = a->nq == NQ6 && !a->overwrite &&
                           (a->assembly == BEMPPCUDA_ASM_EFIE || a->assembly == BEMPPCUDA_ASM_MFIE) &&
                           a->kernel == BEMPPCUDA_HELMHOLTZ_SLP && a->params[0] > 0.0 &&
                           a->test.shapeset == BEMPPCUDA_SHAPE_RWG && a->trial.shapeset == BEMPPCUDA_SHAPE_RWG &&
                           a->test.nshape == 3 && a->trial.nshape == 3;
    if (a->precision == BEMPPCUDA_MIXED && !dp0 && !p1_mixed && !rwg_mixed) {
        bc_set_error("mixed precision is implemented for DP0 scalar kernels, the P1 single, double, adjoint "
                     "double layer and hypersingular operators (Helmholtz with Re k > 0, Laplace, modified "
                     "Helmholtz) and the Maxwell electric and magnetic fields (Re k > 0), with the 6-point rule");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    cudaError_t err = cudaSuccess;
    const int mixed = a->precision == BEMPPCUDA_MIXED;
    // the phase k (r - r_c) is bounded by |k| (R_test + R_trial): at most 1 or
    // 1/2 lets the sine / cosine skip the range reduction (classes 1, 2)
    const double theta = fabs(a->params[0]) * a->phase_radius;
    const int phase_class = a->phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
    // one DP0 space on both sides of one grid: each element pair gives A_ij and A_ji
    const bool sym = dp0 && !a->no_symmetry && a->grids_identical && a->test.support == a->trial.support &&
                     a->test.nsupport == a->trial.nsupport && a->test_grid.geom == a->trial_grid.geom &&
                     a->test.normal_mult == a->trial.normal_mult && prm.ntest == prm.ntrial;
    const bool ranged = a->row_begin != 0 || a->row_end != 0;
    // the kernels with a symmetric sweep, and its wavenumber condition (launch_dp0)
    const bool laplace = a->kernel <= BEMPPCUDA_LAPLACE_ADLP;
    const bool modhelm = a->kernel >= BEMPPCUDA_MODHELM_SLP && a->kernel <= BEMPPCUDA_MODHELM_ADLP;
    const bool sym_kernel = laplace || modhelm || a->kernel == BEMPPCUDA_HELMHOLTZ_SLP ||
                            a->kernel == BEMPPCUDA_HELMHOLTZ_DLP || a->kernel == BEMPPCUDA_HELMHOLTZ_ADLP ||
                            a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED;
    const bool sym_ok = sym && sym_kernel &&
                        (laplace || a->precision != BEMPPCUDA_MIXED || a->params[0] > 0.0);
    if (ranged && (!sym_ok || a->row_begin < 0 || a->row_end > prm.ntest || a->row_begin >= a->row_end)) {
        bc_set_error("row range [%lld, %lld) needs the symmetric sweep and 0 <= begin < end <= %lld rows",
                     (long long)a->row_begin, (long long)a->row_end, (long long)prm.ntest);
        return BEMPPCUDA_ERR_INVALID;
    }
    const int64_t row0 = ranged ? a->row_begin : 0, row1 = ranged ? a->row_end : prm.ntest;
    if (a->tresult) {
        // stripe mode: only the DP0 symmetric sweep over a row range stores into local buffers
        if (!ranged || !dp0 || !sym_ok || a->col_begin < 0 || a->col_begin > a->row_begin ||
            a->ld < prm.ntrial - a->col_begin) {
            bc_set_error("tresult needs the DP0 symmetric sweep over a row range, 0 <= col_begin <= row_begin "
                         "and ld >= columns - col_begin");
            return BEMPPCUDA_ERR_INVALID;
        }
        const bool kernel_ok = a->kernel == BEMPPCUDA_HELMHOLTZ_SLP || a->kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
                               a->kernel == BEMPPCUDA_HELMHOLTZ_ADLP || a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED ||
                               a->kernel == BEMPPCUDA_LAPLACE_SLP;
        if (!kernel_ok) {
            bc_set_error("tresult (stripe mode): Helmholtz single, double, adjoint double layer, combined field "
                         "and Laplace single layer only");
            return BEMPPCUDA_ERR_UNSUPPORTED;
        }
        prm.tresult = a->tresult;
        prm.row0 = a->row_begin;
        prm.col0 = a->col_begin;
    }
    if (dp0) {
        switch (a->kernel) {
        case BEMPPCUDA_LAPLACE_SLP: err = launch_dp0<BEMPPCUDA_LAPLACE_SLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_LAPLACE_DLP: err = launch_dp0<BEMPPCUDA_LAPLACE_DLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_LAPLACE_ADLP: err = launch_dp0<BEMPPCUDA_LAPLACE_ADLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_MODHELM_SLP: err = launch_dp0<BEMPPCUDA_MODHELM_SLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_MODHELM_DLP: err = launch_dp0<BEMPPCUDA_MODHELM_DLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_MODHELM_ADLP: err = launch_dp0<BEMPPCUDA_MODHELM_ADLP>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_dp0<BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, mixed, phase_class, sym, row0, row1, st); break;
        default: bc_set_error("kernel %d not valid for boundary assembly", a->kernel); return BEMPPCUDA_ERR_INVALID;
        }
    } else if ((a->assembly == BEMPPCUDA_ASM_EFIE || a->assembly == BEMPPCUDA_ASM_MFIE) && a->nq == NQ6 &&
               !a->overwrite && a->kernel == BEMPPCUDA_HELMHOLTZ_SLP && (a->params[0] != 0.0 || a->params[1] != 0.0) &&
               a->test.shapeset == BEMPPCUDA_SHAPE_RWG && a->trial.shapeset == BEMPPCUDA_SHAPE_RWG &&
               a->test.nshape == 3 && a->trial.nshape == 3) {
        // RWG and SNC share their dof maps; the caller passes the same arrays for both
        const bool rsym = !a->no_symmetry && a->grids_identical && a->test.support == a->trial.support &&
                          a->test.l2g == a->trial.l2g && a->test.mult == a->trial.mult &&
                          a->test.nsupport == a->trial.nsupport && a->test_grid.geom == a->trial_grid.geom &&
                          prm.ntest == prm.ntrial;
        // a complex wavenumber takes phase class 3 (exp(-Im k r) per point pair)
        const int rwg_phase = a->params[1] != 0.0 ? 3 : phase_class;
        if (mixed && rwg_mixed && a->assembly == BEMPPCUDA_ASM_EFIE)
            err = launch_p1_mixed<BEMPPCUDA_ASM_EFIE, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, phase_class, rsym, st);
        else if (mixed && rwg_mixed)
            err = launch_p1_mixed<BEMPPCUDA_ASM_MFIE, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, phase_class, rsym, st);
        else if (a->assembly == BEMPPCUDA_ASM_EFIE)
            err = launch_rwg<BEMPPCUDA_ASM_EFIE>(prm, rule, rwg_phase, rsym, st);
        else
            err = launch_rwg<BEMPPCUDA_ASM_MFIE>(prm, rule, rwg_phase, rsym, st);
    } else if (const bool psym = !a->no_symmetry && a->grids_identical && a->test.support == a->trial.support &&
                                 a->test.l2g == a->trial.l2g && a->test.mult == a->trial.mult &&
                                 a->test.nsupport == a->trial.nsupport && a->test_grid.geom == a->trial_grid.geom &&
                                 a->test.normal_mult == a->trial.normal_mult && prm.ntest == prm.ntrial;
               a->nq == NQ6 && !a->overwrite && a->test.shapeset != BEMPPCUDA_SHAPE_RWG &&
               a->trial.shapeset != BEMPPCUDA_SHAPE_RWG &&
               ((a->assembly == BEMPPCUDA_ASM_SCALAR && a->kernel <= BEMPPCUDA_MODHELM_ADLP) ||
                a->assembly == BEMPPCUDA_ASM_LAPLACE_HYP || a->assembly == BEMPPCUDA_ASM_HELM_HYP ||
                a->assembly == BEMPPCUDA_ASM_MODHELM_HYP)) {
        // single layer / hypersingular on one space into a zeroed result: the pairs i < j add their
        // blocks U, then A = U + U^T (the regular diagonal is zero), half the global atomics
        const bool defer = psym && a->result_is_zero && a->test.nshape == a->trial.nshape &&
                           a->test.ndofs == a->trial.ndofs && a->test.ndofs <= 32 * 65535LL &&
                           (a->assembly != BEMPPCUDA_ASM_SCALAR || a->kernel == BEMPPCUDA_LAPLACE_SLP ||
                            a->kernel == BEMPPCUDA_HELMHOLTZ_SLP || a->kernel == BEMPPCUDA_MODHELM_SLP);
        prm.defer_transpose = defer ? 1 : 0;
        // a complex wavenumber takes phase class 3 (no centroid factoring, exp(-Im k r) per point)
        const int p1_phase = a->params[1] != 0.0 ? 3 : phase_class;
        if (mixed && p1_mixed) {
            if (a->assembly == BEMPPCUDA_ASM_HELM_HYP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_HELM_HYP, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, phase_class, psym, st);
            else if (a->assembly == BEMPPCUDA_ASM_LAPLACE_HYP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_LAPLACE_HYP, BEMPPCUDA_LAPLACE_SLP>(prm, rule, 0, psym, st);
            else if (a->assembly == BEMPPCUDA_ASM_MODHELM_HYP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_MODHELM_HYP, BEMPPCUDA_MODHELM_SLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_LAPLACE_SLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_LAPLACE_SLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_LAPLACE_DLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_LAPLACE_DLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_LAPLACE_ADLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_LAPLACE_ADLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_MODHELM_SLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_MODHELM_SLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_MODHELM_DLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_MODHELM_DLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_MODHELM_ADLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_MODHELM_ADLP>(prm, rule, 0, psym, st);
            else if (a->kernel == BEMPPCUDA_HELMHOLTZ_DLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, phase_class, psym, st);
            else if (a->kernel == BEMPPCUDA_HELMHOLTZ_ADLP)
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, phase_class, psym, st);
            else
                err = launch_p1_mixed<BEMPPCUDA_ASM_SCALAR, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, phase_class, psym, st);
        } else if (a->assembly == BEMPPCUDA_ASM_LAPLACE_HYP) {
            err = launch_p1<BEMPPCUDA_ASM_LAPLACE_HYP, BEMPPCUDA_LAPLACE_SLP>(prm, rule, p1_phase, psym, st);
        } else if (a->assembly == BEMPPCUDA_ASM_HELM_HYP) {
            err = launch_p1<BEMPPCUDA_ASM_HELM_HYP, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, p1_phase, psym, st);
        } else if (a->assembly == BEMPPCUDA_ASM_MODHELM_HYP) {
            err = launch_p1<BEMPPCUDA_ASM_MODHELM_HYP, BEMPPCUDA_MODHELM_SLP>(prm, rule, p1_phase, psym, st);
        } else {
            switch (a->kernel) {
            case BEMPPCUDA_LAPLACE_SLP: err = launch_p1<0, BEMPPCUDA_LAPLACE_SLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_LAPLACE_DLP: err = launch_p1<0, BEMPPCUDA_LAPLACE_DLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_LAPLACE_ADLP: err = launch_p1<0, BEMPPCUDA_LAPLACE_ADLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_p1<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_p1<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_p1<0, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_MODHELM_SLP: err = launch_p1<0, BEMPPCUDA_MODHELM_SLP>(prm, rule, p1_phase, psym, st); break;
            case BEMPPCUDA_MODHELM_DLP: err = launch_p1<0, BEMPPCUDA_MODHELM_DLP>(prm, rule, p1_phase, psym, st); break;
            default: err = launch_p1<0, BEMPPCUDA_MODHELM_ADLP>(prm, rule, p1_phase, psym, st); break;
            }
        }
        if (defer && err == cudaSuccess) err = launch_add_transpose(prm.result, a->test.ndofs, prm.ld, prm.is_complex, st);
    } else {
        switch (a->assembly) {
        case BEMPPCUDA_ASM_SCALAR:
            switch (a->kernel) {
            case BEMPPCUDA_LAPLACE_SLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_SLP>(prm, rule, st); break;
            case BEMPPCUDA_LAPLACE_DLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_DLP>(prm, rule, st); break;
            case BEMPPCUDA_LAPLACE_ADLP: err = launch_generic<0, BEMPPCUDA_LAPLACE_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_SLP: err = launch_generic<0, BEMPPCUDA_MODHELM_SLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_DLP: err = launch_generic<0, BEMPPCUDA_MODHELM_DLP>(prm, rule, st); break;
            case BEMPPCUDA_MODHELM_ADLP: err = launch_generic<0, BEMPPCUDA_MODHELM_ADLP>(prm, rule, st); break;
            case BEMPPCUDA_HELMHOLTZ_COMBINED: err = launch_generic<0, BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, st); break;
            default: bc_set_error("kernel %d not valid for boundary assembly", a->kernel); return BEMPPCUDA_ERR_INVALID;
            }
            break;
        case BEMPPCUDA_ASM_LAPLACE_HYP: err = launch_generic<1, BEMPPCUDA_LAPLACE_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_HELM_HYP: err = launch_generic<2, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_MODHELM_HYP: err = launch_generic<3, BEMPPCUDA_MODHELM_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_EFIE: err = launch_generic<4, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        case BEMPPCUDA_ASM_MFIE: err = launch_generic<5, BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, st); break;
        default: bc_set_error("assembly type %d unknown", a->assembly); return BEMPPCUDA_ERR_INVALID;
        }
    }
    if (err != cudaSuccess) {
        bc_set_error("regular assembly launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
