// Matrix-free FP64 operator apply: y += A_reg x for one DP0 space of one grid,
// A_reg the regular (non-adjacent) part of the Galerkin matrix, evaluated on
// the fly and never stored.
//
// Used for the residual b - A x of the mixed-precision refinement: the mixed
// matrix holds FP32-evaluated regular pairs, so residuals formed with it
// converge to the mixed operator's solution; residuals formed with this
// apply (plus the FP64 singular / identity entries, which the mixed matrix
// holds exactly) converge to the FP64 operator's solution.
//
// The sweep is the FP64 symmetric tile of the assembly (dp0_sym.cuh: one pass
// over the 36 point pairs of (i, j), i < j, gives A_ij and A_ji); instead of
// storing the two entries a thread adds A_ji x_i to its column sum (one
// atomic per thread and tile) and A_ij x_j is summed over the warp's 32
// columns with shuffles (one atomic per warp and row).  Same arithmetic per
// entry as the assembly, different summation order.
#include "common.cuh"
#include "dp0_sym.cuh"

namespace bc {

__device__ __forceinline__ double warp_sum64(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// blockIdx.x = column block of 128 trial elements, blockIdx.y = row chunk of tile_rows test
// elements; chunks below the block's last column have no pair i < j and exit at once.  Every
// lane of a warp runs every row step (the shuffles need the whole warp).
template <int K, int PHC>
__global__ void __launch_bounds__(DP0_THREADS) regular_dp0_apply64(RegParams prm, QuadRule rule,
                                                                   const double2 *__restrict__ x, double2 *y,
                                                                   int tile_rows) {
    const int64_t t0 = (int64_t)blockIdx.y * tile_rows;
    if (t0 >= ((int64_t)blockIdx.x + 1) * DP0_THREADS) return;
    __shared__ TestBlock64s sb;
    const int tcount = (int)min((int64_t)tile_rows, prm.ntest - t0);
    stage_sym64(prm, rule, t0, tcount, sb);
    __syncthreads();

    const int64_t si = (int64_t)blockIdx.x * DP0_THREADS + threadIdx.x;
    const bool column = si < prm.ntrial && t0 < si;
    SymTrial64 tr;
    double2 xj = make_double2(0.0, 0.0);
    if (column) {
        load_trial_sym64<K, PHC>(prm, rule, si, tr);
        xj = x[si];
    }
    double yr = 0.0, yi = 0.0;  // sum over the block's rows i of A_ji x_i (column j = si)
    for (int tt = 0; tt < tcount; ++tt) {
        const int64_t row = t0 + tt;
        double cr = 0.0, ci = 0.0;  // A_ij x_j
        // row < si: the pairs above the diagonal; adjacent pairs (and i = j) belong to the singular part
        if (column && row < si && !(prm.grids_identical && shares_vertex(sb.v[tt], tr.sv0, tr.sv1, tr.sv2))) {
            double a_re, a_im, b_re, b_im;
            pair_sym64<K, PHC>(prm, rule, sb, tt, tr, a_re, a_im, b_re, b_im);
            cr = fma(a_re, xj.x, -a_im * xj.y);
            ci = fma(a_re, xj.y, a_im * xj.x);
            const double2 xi = x[row];
            yr += fma(b_re, xi.x, -b_im * xi.y);
            yi += fma(b_re, xi.y, b_im * xi.x);
        }
        if (__any_sync(0xffffffffu, cr != 0.0 || ci != 0.0)) {
            cr = warp_sum64(cr);
            ci = warp_sum64(ci);
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(&y[row].x, cr);
                atomicAdd(&y[row].y, ci);
            }
        }
    }
    if (column && (yr != 0.0 || yi != 0.0)) {
        atomicAdd(&y[si].x, yr);
        atomicAdd(&y[si].y, yi);
    }
}

template <int K>
static cudaError_t launch_apply(const RegParams &prm, const QuadRule &rule, int phase_class, const double2 *x,
                                double2 *y, cudaStream_t st) {
    const unsigned bx = (unsigned)((prm.ntrial + DP0_THREADS - 1) / DP0_THREADS);
    // rows per tile as in the assembly's symmetric sweep: fewer when 32-row tiles leave the GPU short of work
    int tile_rows = DP0_TCHUNK;
    const int64_t wave = (int64_t)bc_sm_count() * 3;
    while (tile_rows > 8 && (int64_t)bx * ((prm.ntest + tile_rows - 1) / tile_rows) / 2 < 4 * wave) tile_rows /= 2;
    const dim3 grid(bx, (unsigned)((prm.ntest + tile_rows - 1) / tile_rows));
    if constexpr (!KernelTraits<K>::helm) {
        regular_dp0_apply64<K, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule, x, y, tile_rows);
    } else {
        if (prm.p[1] != 0.0)
            regular_dp0_apply64<K, 3><<<grid, DP0_THREADS, 0, st>>>(prm, rule, x, y, tile_rows);
        else if (phase_class == 2)
            regular_dp0_apply64<K, 2><<<grid, DP0_THREADS, 0, st>>>(prm, rule, x, y, tile_rows);
        else if (phase_class == 1)
            regular_dp0_apply64<K, 1><<<grid, DP0_THREADS, 0, st>>>(prm, rule, x, y, tile_rows);
        else
            regular_dp0_apply64<K, 0><<<grid, DP0_THREADS, 0, st>>>(prm, rule, x, y, tile_rows);
    }
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

// Validated arguments in (capi.cu), launch out.
int bc_apply_launch(const bemppcuda_regular_args *a, const void *x, void *y, cudaStream_t st) {
    const bool dp0 = a->assembly == BEMPPCUDA_ASM_SCALAR && a->test.nshape == 1 && a->trial.nshape == 1 &&
                     a->test.dof_is_position && a->trial.dof_is_position && a->nq == NQ6;
    const bool same = a->grids_identical && a->test.support == a->trial.support &&
                      a->test.nsupport == a->trial.nsupport && a->test_grid.geom == a->trial_grid.geom &&
                      a->test.normal_mult == a->trial.normal_mult;
    const bool kernel_ok = a->kernel == BEMPPCUDA_LAPLACE_SLP || a->kernel == BEMPPCUDA_LAPLACE_DLP ||
                           a->kernel == BEMPPCUDA_LAPLACE_ADLP || a->kernel == BEMPPCUDA_HELMHOLTZ_SLP ||
                           a->kernel == BEMPPCUDA_HELMHOLTZ_DLP || a->kernel == BEMPPCUDA_HELMHOLTZ_ADLP ||
                           a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED;
    if (!dp0 || !same || !kernel_ok || a->precision != BEMPPCUDA_FP64) {
        bc_set_error("apply_regular: FP64 Laplace / Helmholtz single, double, adjoint double layer or combined "
                     "field on one DP0 space of one grid (identity dof map, 6-point rule) only");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    RegParams prm = {};
    prm.tg = prm.sg = a->test_grid.geom;
    prm.tne = prm.sne = a->test_grid.nelements;
    prm.tel = prm.sel = a->test_grid.elements;
    prm.tsup = a->test.support;
    prm.ssup = a->trial.support;
    prm.ntest = a->test.nsupport;
    prm.ntrial = a->trial.nsupport;
    prm.tnm = a->test.normal_mult;
    prm.snm = a->trial.normal_mult;
    prm.tnshape = prm.snshape = 1;
    prm.grids_identical = 1;
    prm.is_complex = 1;
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    if (prm.ntest == 0) return BEMPPCUDA_OK;
    QuadRule rule;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);
    const double theta = fabs(a->params[0]) * a->phase_radius;
    const int phase_class = a->phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
    const double2 *xv = reinterpret_cast<const double2 *>(x);
    double2 *yv = reinterpret_cast<double2 *>(y);
    cudaError_t err;
    switch (a->kernel) {
    case BEMPPCUDA_LAPLACE_SLP: err = launch_apply<BEMPPCUDA_LAPLACE_SLP>(prm, rule, phase_class, xv, yv, st); break;
    case BEMPPCUDA_LAPLACE_DLP: err = launch_apply<BEMPPCUDA_LAPLACE_DLP>(prm, rule, phase_class, xv, yv, st); break;
    case BEMPPCUDA_LAPLACE_ADLP: err = launch_apply<BEMPPCUDA_LAPLACE_ADLP>(prm, rule, phase_class, xv, yv, st); break;
    case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_apply<BEMPPCUDA_HELMHOLTZ_SLP>(prm, rule, phase_class, xv, yv, st); break;
    case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_apply<BEMPPCUDA_HELMHOLTZ_DLP>(prm, rule, phase_class, xv, yv, st); break;
    case BEMPPCUDA_HELMHOLTZ_ADLP: err = launch_apply<BEMPPCUDA_HELMHOLTZ_ADLP>(prm, rule, phase_class, xv, yv, st); break;
    default: err = launch_apply<BEMPPCUDA_HELMHOLTZ_COMBINED>(prm, rule, phase_class, xv, yv, st); break;
    }
    if (err != cudaSuccess) {
        bc_set_error("apply_regular: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
