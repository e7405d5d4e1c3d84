// Batched DP0 assembly: many grids and wavenumbers in one persistent launch.
//
// The work list is every (problem, tile) pair, tile = rows_per_item (<= 32)
// test x 128 trial elements of one problem's matrix.  A persistent grid (blocks_per_sm x SMs
// CTAs) pulls items from a global atomic counter, so uneven problems (512 to
// 8192 elements here) balance dynamically; each item runs the same tile code
// as the single-problem kernels (dp0.cuh) with that problem's parameters and
// precision.  The singular pairs of all problems go through one warp-per-pair
// launch over the concatenated pair list (FP64).
#include <cstring>

#include "dp0_sym.cuh"
#include "singular_dp0.cuh"

namespace bc {

struct BatchDev {
    RegParams prm;
    int64_t tile_begin;
    int64_t tiles_x;
    int32_t rows;  // test elements per work item (<= DP0_TCHUNK)
    int32_t sym;   // symmetric sweep: items cover the tiles on or above the diagonal
    int64_t pair_begin;
    int32_t precision;
    int32_t phase_class;
    int32_t ck;
    int32_t pad;
    double diag_shift;
};

constexpr size_t kCounterBytes = 256;

union TileShared {
    TestBlock64 b64;
    TestBlock64s b64s;
    TestBlock32 b32;
    TestBlock32p b32p;
    TestBlock32q b32q;
};

template <int K>
__device__ __forceinline__ void run_tile(const BatchDev &P, const QuadRule &rule, int64_t tx, int64_t ty,
                                         TileShared &sh) {
    const int64_t t0 = ty * P.rows;
    const int rows = P.rows;
    if (P.precision == BEMPPCUDA_FP64) {
        if (P.ck)
            regular_dp0_fp64_tile<K, true, 0>(P.prm, rule, tx, t0, rows, sh.b64);
        else if (P.phase_class == 2)
            regular_dp0_fp64_tile<K, false, 2>(P.prm, rule, tx, t0, rows, sh.b64);
        else if (P.phase_class == 1)
            regular_dp0_fp64_tile<K, false, 1>(P.prm, rule, tx, t0, rows, sh.b64);
        else
            regular_dp0_fp64_tile<K, false, 0>(P.prm, rule, tx, t0, rows, sh.b64);
    } else {
        if (P.ck)
            regular_dp0_mixed_tile<K, true, 0>(P.prm, rule, tx, t0, rows, sh.b32);
        else if (!(P.prm.p[0] > 0.0))  // the packed path needs k > 0
            regular_dp0_mixed_tile<K, false, 0>(P.prm, rule, tx, t0, rows, sh.b32);
        else if (P.phase_class == 2)
            regular_dp0_mixed2_tile<K, 2>(P.prm, rule, tx, t0, rows, sh.b32p);
        else if (P.phase_class == 1)
            regular_dp0_mixed2_tile<K, 1>(P.prm, rule, tx, t0, rows, sh.b32p);
        else
            regular_dp0_mixed2_tile<K, 0>(P.prm, rule, tx, t0, rows, sh.b32p);
    }
}

// Symmetric sweep of one problem (Re k > 0 on the mixed path; a complex k is phase class 3 of the FP64
// tile and the amplitude split of the mixed one): tile (tx, ty) = columns [128 tx, 128 tx + 128) x rows
// [rows ty, rows ty + rows).
template <int K>
__device__ __forceinline__ void run_tile_sym(const BatchDev &P, const QuadRule &rule, int64_t tx, int64_t ty,
                                             TileShared &sh) {
    const int64_t t0 = ty * P.rows;
    const int rows = P.rows;
    if (P.precision == BEMPPCUDA_FP64) {
        if (KernelTraits<K>::helm && P.ck)
            regular_dp0_fp64_sym_tile<K, 3>(P.prm, rule, tx, t0, rows, sh.b64s);
        else if (P.phase_class == 2)
            regular_dp0_fp64_sym_tile<K, 2>(P.prm, rule, tx, t0, rows, sh.b64s);
        else if (P.phase_class == 1)
            regular_dp0_fp64_sym_tile<K, 1>(P.prm, rule, tx, t0, rows, sh.b64s);
        else
            regular_dp0_fp64_sym_tile<K, 0>(P.prm, rule, tx, t0, rows, sh.b64s);
    } else if constexpr (KernelTraits<K>::helm) {
        if (P.ck) {
            if (P.phase_class == 2)
                regular_dp0_mixed_sym_tile<K, 2, false, true>(P.prm, rule, tx, t0, rows, sh.b32q);
            else if (P.phase_class == 1)
                regular_dp0_mixed_sym_tile<K, 1, false, true>(P.prm, rule, tx, t0, rows, sh.b32q);
            else
                regular_dp0_mixed_sym_tile<K, 0, false, true>(P.prm, rule, tx, t0, rows, sh.b32q);
        } else if (P.phase_class == 2) {
            regular_dp0_mixed_sym_tile<K, 2>(P.prm, rule, tx, t0, rows, sh.b32q);
        } else if (P.phase_class == 1) {
            regular_dp0_mixed_sym_tile<K, 1>(P.prm, rule, tx, t0, rows, sh.b32q);
        } else {
            regular_dp0_mixed_sym_tile<K, 0>(P.prm, rule, tx, t0, rows, sh.b32q);
        }
    } else {
        regular_dp0_mixed_sym_tile<K, 0>(P.prm, rule, tx, t0, rows, sh.b32q);
    }
}

// Tiles before column tx of a symmetric problem: column u holds g (u + 1)
// row tiles (g = 128 / rows), clipped to the row-tile count only in the last column.
__host__ __device__ __forceinline__ int64_t sym_tiles_before(int64_t tx, int64_t g) { return g * tx * (tx + 1) / 2; }

__device__ __forceinline__ void sym_coords(const BatchDev &P, int64_t local, int64_t *tx, int64_t *ty) {
    const int64_t g = DP0_THREADS / P.rows;
    int64_t c = (int64_t)((sqrt(1.0 + 8.0 * (double)local / (double)g) - 1.0) * 0.5);
    while (c > 0 && sym_tiles_before(c, g) > local) --c;
    while (c + 1 < P.tiles_x && sym_tiles_before(c + 1, g) <= local) ++c;
    *tx = c;
    *ty = local - sym_tiles_before(c, g);
}

// Index of the last problem whose range starts at or before `item`.
__device__ __forceinline__ int find_problem(const BatchDev *__restrict__ probs, int nprob, int64_t item,
                                            bool by_pairs) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int64_t begin = by_pairs ? probs[mid].pair_begin : probs[mid].tile_begin;
        if (begin <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int K>
__global__ void __launch_bounds__(DP0_THREADS) regular_batch(const BatchDev *__restrict__ probs, int nprob,
                                                              int64_t total_tiles,
                                                              unsigned long long *__restrict__ counter,
                                                              QuadRule rule) {
    __shared__ TileShared sh;
    __shared__ long long s_tile;
    while (true) {
        if (threadIdx.x == 0) s_tile = (long long)atomicAdd(counter, 1ull);
        __syncthreads();
        const int64_t tile = s_tile;
        __syncthreads();
        if (tile >= total_tiles) break;
        const BatchDev &P = probs[find_problem(probs, nprob, tile, false)];
        const int64_t local = tile - P.tile_begin;
        if (P.sym) {
            int64_t tx, ty;
            sym_coords(P, local, &tx, &ty);
            run_tile_sym<K>(P, rule, tx, ty, sh);
        } else {
            run_tile<K>(P, rule, local % P.tiles_x, local / P.tiles_x, sh);
        }
    }
}

struct SingBatchTables {
    const double *tp, *sp, *w;
    const uint32_t *te, *se, *toff, *soff, *woff, *npts;
    int64_t npairs;
};

constexpr int SB_WARPS = 8;

// One warp per singular pair of any problem (DP0 spaces: the pair's entry is
// row = test element, column = trial element of that problem).
template <int K>
__global__ void __launch_bounds__(32 * SB_WARPS) singular_batch(const BatchDev *__restrict__ probs, int nprob,
                                                                 SingBatchTables tab) {
    const int lane = threadIdx.x & 31;
    const int64_t k = (int64_t)blockIdx.x * SB_WARPS + (threadIdx.x >> 5);
    if (k >= tab.npairs) return;
    const BatchDev &P = probs[find_problem(probs, nprob, k, true)];
    const RegParams &prm = P.prm;
    const int64_t t = tab.te[k], s = tab.se[k];
    Geom gt, gs;
    load_geom(prm.tg, prm.tne, t, 1.0, gt);
    load_geom(prm.tg, prm.tne, s, 1.0, gs);
    double vr = 0.0, vi = 0.0;
    const double2 *tp = reinterpret_cast<const double2 *>(tab.tp), *sp = reinterpret_cast<const double2 *>(tab.sp);
    const int64_t toff = tab.toff[k], soff = tab.soff[k], woff = tab.woff[k];
    const int n = (int)tab.npts[k];
    if (P.ck)
        sing_dp0_value<K, 3>(prm.tg, prm.tne, t, s, gt, gs, prm.p, tp, sp, tab.w, toff, soff, woff, n, &vr, &vi);
    else if (P.phase_class == 2)
        sing_dp0_value<K, 2>(prm.tg, prm.tne, t, s, gt, gs, prm.p, tp, sp, tab.w, toff, soff, woff, n, &vr, &vi);
    else if (P.phase_class == 1)
        sing_dp0_value<K, 1>(prm.tg, prm.tne, t, s, gt, gs, prm.p, tp, sp, tab.w, toff, soff, woff, n, &vr, &vi);
    else
        sing_dp0_value<K, 0>(prm.tg, prm.tne, t, s, gt, gs, prm.p, tp, sp, tab.w, toff, soff, woff, n, &vr, &vi);
    vr *= BC_INV_4PI;
    vi *= BC_INV_4PI;
    if (lane == 0) {
        const double scale = gt.ie * gs.ie;
        vr *= scale;
        vi *= scale;
        if (t == s) vr += P.diag_shift * 0.5 * gt.ie;
        double2 *o = reinterpret_cast<double2 *>(prm.result) + t * prm.ld + s;
        const double2 old = *o;
        *o = make_double2(old.x + vr, old.y + vi);
    }
}

}  // namespace bc

using namespace bc;

static int64_t tiles_of(int64_t n, int rows, bool sym) {
    const int64_t tx = (n + DP0_THREADS - 1) / DP0_THREADS, ty = (n + rows - 1) / rows;
    if (!sym || tx == 0) return tx * ty;
    const int64_t g = DP0_THREADS / rows;
    return sym_tiles_before(tx - 1, g) + (ty < g * tx ? ty : g * tx);
}

static int rows_of(const bemppcuda_batch_args *a) {
    return (a->rows_per_item >= 1 && a->rows_per_item <= DP0_TCHUNK) ? a->rows_per_item : DP0_TCHUNK;
}

// The symmetric sweep needs Re k > 0 on the scaled mixed path (a complex k included) and a row height
// that divides the 128-column block.
static bool sym_of(const bemppcuda_batch_problem &p, int rows) {
    if (DP0_THREADS % rows != 0) return false;
    return p.precision == BEMPPCUDA_FP64 || p.params[0] > 0.0;
}

extern "C" int64_t bemppcuda_batch_workspace_bytes(int32_t nproblems) {
    if (nproblems < 0) return 0;
    return (int64_t)kCounterBytes + (int64_t)nproblems * (int64_t)sizeof(BatchDev);
}

static int batch_check(const bemppcuda_batch_args *a) {
    if (!a || !a->problems || a->nproblems <= 0) {
        bc_set_error("batch: problem list missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->kernel != BEMPPCUDA_HELMHOLTZ_SLP && a->kernel != BEMPPCUDA_HELMHOLTZ_COMBINED) {
        bc_set_error("batch: kernel must be BEMPPCUDA_HELMHOLTZ_SLP or BEMPPCUDA_HELMHOLTZ_COMBINED");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    if (a->nq != 6 || !a->quad_points || !a->quad_weights) {
        bc_set_error("batch: the 6-point regular rule is required");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (!a->workspace || a->workspace_bytes < bemppcuda_batch_workspace_bytes(a->nproblems)) {
        bc_set_error("batch: workspace too small");
        return BEMPPCUDA_ERR_WORKSPACE;
    }
    int64_t pairs = 0;
    for (int i = 0; i < a->nproblems; ++i) {
        const bemppcuda_batch_problem &p = a->problems[i];
        if (!p.grid.geom || !p.grid.elements || !p.support || !p.result || p.grid.nelements <= 0 ||
            p.ld < p.grid.nelements) {
            bc_set_error("batch: problem %d is incomplete", i);
            return BEMPPCUDA_ERR_INVALID;
        }
        if (p.precision != BEMPPCUDA_FP64 && p.precision != BEMPPCUDA_MIXED) {
            bc_set_error("batch: problem %d has an unknown precision", i);
            return BEMPPCUDA_ERR_INVALID;
        }
        if (p.pair_begin != pairs || p.pair_count < 0) {
            bc_set_error("batch: the singular pairs of problem %d must directly follow those of the previous one", i);
            return BEMPPCUDA_ERR_INVALID;
        }
        for (int j = 0; j < 4; ++j)
            if (!(p.params[j] == p.params[j])) {
                bc_set_error("batch: problem %d has a non-finite parameter", i);
                return BEMPPCUDA_ERR_INVALID;
            }
        pairs += p.pair_count;
    }
    if (pairs != a->npairs || (pairs > 0 && (!a->test_points || !a->trial_points || !a->weights ||
                                              !a->test_elements || !a->trial_elements || !a->test_offsets ||
                                              !a->trial_offsets || !a->weights_offsets || !a->npoints))) {
        bc_set_error("batch: the singular pair arrays do not match the problem list");
        return BEMPPCUDA_ERR_INVALID;
    }
    return BEMPPCUDA_OK;
}

extern "C" int bemppcuda_batch_prepare(const bemppcuda_batch_args *a, void *stream) {
    int rc = batch_check(a);
    if (rc) return rc;
    BatchDev *host = new BatchDev[a->nproblems];
    int64_t tiles = 0;
    for (int i = 0; i < a->nproblems; ++i) {
        const bemppcuda_batch_problem &p = a->problems[i];
        BatchDev &d = host[i];
        memset(&d, 0, sizeof(d));
        RegParams &r = d.prm;
        r.tg = r.sg = p.grid.geom;
        r.tne = r.sne = p.grid.nelements;
        r.tel = r.sel = p.grid.elements;
        r.tsup = r.ssup = p.support;
        r.ntest = r.ntrial = p.grid.nelements;
        r.tnshape = r.snshape = 1;
        r.grids_identical = 1;
        r.is_complex = 1;
        r.overwrite = 1;
        for (int j = 0; j < 4; ++j) r.p[j] = p.params[j];
        r.result = p.result;
        r.ld = p.ld;
        d.tile_begin = tiles;
        d.tiles_x = (p.grid.nelements + DP0_THREADS - 1) / DP0_THREADS;
        d.rows = rows_of(a);
        d.sym = sym_of(p, d.rows) ? 1 : 0;
        tiles += tiles_of(p.grid.nelements, d.rows, d.sym != 0);
        d.pair_begin = p.pair_begin;
        d.precision = p.precision;
        r.near_r = p.phase_radius > 0.0 ? p.phase_radius : 0.0;  // 2 R bounds adjacent centroid distances
        const double theta = fabs(p.params[0]) * p.phase_radius;
        d.phase_class = p.phase_radius > 0.0 ? (theta <= 0.5 ? 2 : (theta <= 1.0 ? 1 : 0)) : 0;
        d.ck = p.params[1] != 0.0;
        d.diag_shift = a->diag_shift;
    }
    char *ws = static_cast<char *>(a->workspace);
    cudaError_t err = cudaMemcpyAsync(ws + kCounterBytes, host, sizeof(BatchDev) * a->nproblems,
                                      cudaMemcpyHostToDevice, (cudaStream_t)stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize((cudaStream_t)stream);
    delete[] host;
    if (err != cudaSuccess) {
        bc_set_error("batch_prepare: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}

template <int K>
static cudaError_t launch_batch(const bemppcuda_batch_args *a, const BatchDev *probs, unsigned long long *counter,
                                int64_t total_tiles, const QuadRule &rule, int blocks, cudaStream_t st) {
    regular_batch<K><<<blocks, DP0_THREADS, 0, st>>>(probs, a->nproblems, total_tiles, counter, rule);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess || a->npairs == 0) return err;
    SingBatchTables tab;
    tab.tp = a->test_points;
    tab.sp = a->trial_points;
    tab.w = a->weights;
    tab.te = a->test_elements;
    tab.se = a->trial_elements;
    tab.toff = a->test_offsets;
    tab.soff = a->trial_offsets;
    tab.woff = a->weights_offsets;
    tab.npts = a->npoints;
    tab.npairs = a->npairs;
    const unsigned sblocks = (unsigned)((a->npairs + SB_WARPS - 1) / SB_WARPS);
    singular_batch<K><<<sblocks, 32 * SB_WARPS, 0, st>>>(probs, a->nproblems, tab);
    return cudaGetLastError();
}

extern "C" int bemppcuda_batch_launch(const bemppcuda_batch_args *a, void *stream) {
    int rc = batch_check(a);
    if (rc) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        bc_set_error("batch_launch: cannot query the device");
        return BEMPPCUDA_ERR_CUDA;
    }
    int64_t total_tiles = 0;
    for (int i = 0; i < a->nproblems; ++i)
        total_tiles += tiles_of(a->problems[i].grid.nelements, rows_of(a), sym_of(a->problems[i], rows_of(a)));
    QuadRule rule;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);
    const int bps = a->blocks_per_sm > 0 ? a->blocks_per_sm : 4;
    const int blocks = bps * sms;
    char *ws = static_cast<char *>(a->workspace);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    const BatchDev *probs = reinterpret_cast<const BatchDev *>(ws + kCounterBytes);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
    if (err == cudaSuccess) {
        if (a->kernel == BEMPPCUDA_HELMHOLTZ_SLP)
            err = launch_batch<BEMPPCUDA_HELMHOLTZ_SLP>(a, probs, counter, total_tiles, rule, blocks, st);
        else
            err = launch_batch<BEMPPCUDA_HELMHOLTZ_COMBINED>(a, probs, counter, total_tiles, rule, blocks, st);
    }
    if (err != cudaSuccess) {
        bc_set_error("batch_launch: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
