// Batched multi-right-hand-side products Y_p = A_p X_p of dense complex128
// operators: the device counterpart of DenseDiscreteBoundaryOperator._matmat
// (api/assembly/discrete_boundary_operator.py:192-198, ndarray.dot on the
// host) for a list of operators with up to 8 right-hand sides each, in one
// launch.
//
// With 8 right-hand sides each 16-byte matrix entry meets 8 complex FMAs
// (64 flops), so the product sits at the FP64 ridge of a B200 (4 flop / byte
// at HBM bandwidth is ~26 TFLOP/s, the FP64 pipe ~36): the kernel must keep
// enough of A in flight to stream it at HBM rate while the FP64 pipe and
// shared memory stay under their limits.  Layout: a CTA of 8 warps owns 16
// rows of one problem (2 rows per warp); columns go in tiles of 64.  A
// three-stage pipeline of asynchronous 16-byte copies (cp.async, L2 only)
// brings each tile of A (16 x 64, 16 KB) and the matching rows of X
// (transposed to xs[c][j], one padding element per row so the transposing
// stores spread over the banks) into shared memory two tiles ahead, about
// 32 KB in flight per CTA.  Each lane reads A(r, j) for its 2 rows and
// j = lane + 32 m, and every X(j, c) once for both rows; one barrier per
// tile.  Partial sums are reduced across the warp with shuffles at the end.
// A CTA's problem is found by binary search over the problems' first row
// blocks.
#include "common.cuh"

namespace bc {

constexpr int MM_THREADS = 256;
constexpr int MM_WARPS = MM_THREADS / 32;
constexpr int MM_RPW = 2;                    // rows per warp
constexpr int MM_ROWS = MM_WARPS * MM_RPW;  // rows per CTA
constexpr int MM_TJ = 64;                    // columns per tile
constexpr int MM_JPL = MM_TJ / 32;           // columns per lane per tile
constexpr int MM_STAGES = 3;                 // tiles in shared memory: one in use, two in flight

struct MatmatDev {
    const double2 *a;
    const double2 *x;
    double2 *y;
    int64_t rows, cols, lda, ldx, ldy;
    int64_t block_begin;
};

// one pipeline stage: a 16 x 64 tile of A and the matching 64 x NR rows of X, transposed
template <int NR>
struct MatmatStage {
    double2 a[MM_ROWS][MM_TJ];
    double2 x[NR][MM_TJ + 1];
};

template <int NR>
constexpr size_t matmat_smem_bytes() {
    return sizeof(MatmatStage<NR>) * MM_STAGES;
}

// The copies a thread issues for every tile: rows r_i = (tid / 64) + 4 i of A at column tid % 64, and
// the X entries e = tid + 256 i (row e / NR, column e % NR of the tile).  Addresses are fixed up to
// the tile offset, so they are formed once per block.
constexpr int MM_ACOPIES = MM_ROWS * MM_TJ / MM_THREADS;
static_assert(MM_THREADS % MM_TJ == 0 && MM_ACOPIES * MM_THREADS == MM_ROWS * MM_TJ, "tile split");

template <int NR>
struct MatmatCopies {
    static constexpr int XC = (NR * MM_TJ + MM_THREADS - 1) / MM_THREADS;
    const double2 *a;        // A(row0 + r_0, tid % 64)
    const double2 *x[XC];    // X(jj_i, c_i)
    int64_t a_step;          // 4 rows of A
    int a_rows;              // rows of the block that exist (<= 16)
    int jj;                  // tid % 64
    int xjj[XC];             // jj_i, or MM_TJ when the thread has no i-th X entry
    unsigned a_dst, x_dst[XC];  // shared-memory offsets within a stage
};

template <int NR>
__device__ __forceinline__ void mm_copies_init(const MatmatDev &P, int64_t row0, MatmatCopies<NR> &cp) {
    const int rb = threadIdx.x / MM_TJ;
    cp.jj = threadIdx.x % MM_TJ;
    cp.a_rows = (int)min((int64_t)MM_ROWS, P.rows - row0);
    cp.a = P.a + min(row0 + rb, P.rows - 1) * P.lda + cp.jj;
    cp.a_step = (int64_t)(MM_THREADS / MM_TJ) * P.lda;
    cp.a_dst = (unsigned)(offsetof(MatmatStage<NR>, a) + (rb * MM_TJ + cp.jj) * sizeof(double2));
#pragma unroll
    for (int i = 0; i < MatmatCopies<NR>::XC; ++i) {
        const int e = threadIdx.x + i * MM_THREADS;
        const int jj = e / NR, c = e - jj * NR;
        cp.xjj[i] = e < NR * MM_TJ ? jj : MM_TJ;
        cp.x[i] = P.x + (e < NR * MM_TJ ? (int64_t)jj * P.ldx + c : 0);
        cp.x_dst[i] = (unsigned)(offsetof(MatmatStage<NR>, x) + (c * (MM_TJ + 1) + jj) * sizeof(double2));
    }
}

// queue the asynchronous copies of tile t (zero fill past the last row / column) and close the group;
// past the last tile the group stays empty, so the wait counts of the main loop hold on every iteration
template <int NR>
__device__ __forceinline__ void mm_stage(const MatmatDev &P, const MatmatCopies<NR> &cp, int64_t t, unsigned base) {
    const int64_t j0 = t * MM_TJ;
    if (j0 < P.cols) {
        const bool jin = j0 + cp.jj < P.cols;
        const double2 *src = cp.a + j0;
#pragma unroll
        for (int i = 0; i < MM_ACOPIES; ++i) {
            const int r = threadIdx.x / MM_TJ + i * (MM_THREADS / MM_TJ);
            const bool in = jin && r < cp.a_rows;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(
                             base + cp.a_dst + (unsigned)(i * (MM_THREADS / MM_TJ) * MM_TJ * sizeof(double2))),
                         "l"(in ? src + i * cp.a_step : P.a), "r"(in ? 16 : 0)
                         : "memory");
        }
        const int64_t xoff = j0 * P.ldx;
#pragma unroll
        for (int i = 0; i < MatmatCopies<NR>::XC; ++i) {
            if (cp.xjj[i] < MM_TJ) {
                const bool in = j0 + cp.xjj[i] < P.cols;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(base + cp.x_dst[i]),
                             "l"(in ? cp.x[i] + xoff : P.x), "r"(in ? 16 : 0)
                             : "memory");
            }
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int NR>
__global__ void __launch_bounds__(MM_THREADS, 2) matmat_c128(const MatmatDev *__restrict__ probs, int nproblems) {
    extern __shared__ __align__(16) unsigned char mm_smem[];
    MatmatStage<NR> *stage = reinterpret_cast<MatmatStage<NR> *>(mm_smem);
    const int64_t b = blockIdx.x;
    int lo = 0, hi = nproblems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (probs[mid].block_begin <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const MatmatDev P = probs[lo];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row0 = (b - P.block_begin) * MM_ROWS;
    double sr[MM_RPW][NR], si[MM_RPW][NR];
#pragma unroll
    for (int r = 0; r < MM_RPW; ++r)
#pragma unroll
        for (int c = 0; c < NR; ++c) sr[r][c] = si[r][c] = 0.0;

    const int64_t ntiles = (P.cols + MM_TJ - 1) / MM_TJ;
    MatmatCopies<NR> cp;
    mm_copies_init<NR>(P, row0, cp);
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(mm_smem);
#pragma unroll
    for (int s = 0; s < MM_STAGES - 1; ++s) mm_stage<NR>(P, cp, s, sbase + s * (unsigned)sizeof(MatmatStage<NR>));
    int cur = 0, nxt = MM_STAGES - 1;  // stages of tile t and of tile t + MM_STAGES - 1
    for (int64_t t = 0; t < ntiles; ++t) {
        asm volatile("cp.async.wait_group %0;\n" ::"n"(MM_STAGES - 2) : "memory");  // tile t has landed
        __syncthreads();  // ... for every thread; and every warp is done with tile t - 1
        mm_stage<NR>(P, cp, t + MM_STAGES - 1, sbase + (unsigned)nxt * (unsigned)sizeof(MatmatStage<NR>));
        const MatmatStage<NR> &s = stage[cur];
        cur = cur == MM_STAGES - 1 ? 0 : cur + 1;
        nxt = nxt == MM_STAGES - 1 ? 0 : nxt + 1;
#pragma unroll
        for (int m = 0; m < MM_JPL; ++m) {
            const int jj = lane + 32 * m;
            double2 a[MM_RPW];
#pragma unroll
            for (int r = 0; r < MM_RPW; ++r) a[r] = s.a[warp * MM_RPW + r][jj];
#pragma unroll
            for (int c = 0; c < NR; ++c) {
                const double2 x = s.x[c][jj];
#pragma unroll
                for (int r = 0; r < MM_RPW; ++r) {
                    sr[r][c] = fma(a[r].x, x.x, fma(-a[r].y, x.y, sr[r][c]));
                    si[r][c] = fma(a[r].x, x.y, fma(a[r].y, x.x, si[r][c]));
                }
            }
        }
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // no copy outlives the block
    // butterfly sums: every lane ends with the totals
#pragma unroll
    for (int r = 0; r < MM_RPW; ++r)
#pragma unroll
        for (int c = 0; c < NR; ++c)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                sr[r][c] += __shfl_xor_sync(0xffffffffu, sr[r][c], off);
                si[r][c] += __shfl_xor_sync(0xffffffffu, si[r][c], off);
            }
    const int64_t rw = row0 + warp * MM_RPW;
#pragma unroll
    for (int r = 0; r < MM_RPW; ++r)
#pragma unroll
        for (int c = 0; c < NR; ++c)
            if (lane == r * NR + c && rw + r < P.rows) P.y[(rw + r) * P.ldy + c] = make_double2(sr[r][c], si[r][c]);
}

}  // namespace bc

using namespace bc;

template <int NR>
static cudaError_t launch_matmat(const MatmatDev *probs, int nproblems, int64_t blocks, cudaStream_t st) {
    constexpr size_t smem = matmat_smem_bytes<NR>();
    // above the 48 KB default: opt in once per device (the attribute is per device and function)
    static std::atomic<int> opted[64];
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 64 && !opted[dev].load()) {
        err = cudaFuncSetAttribute(matmat_c128<NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err != cudaSuccess) return err;
        opted[dev].store(1);
    }
    matmat_c128<NR><<<dim3((unsigned)blocks), MM_THREADS, smem, st>>>(probs, nproblems);
    return cudaGetLastError();
}

extern "C" int64_t bemppcuda_matmat_workspace_bytes(int32_t nproblems) {
    if (nproblems < 0) return 0;
    return (int64_t)nproblems * (int64_t)sizeof(MatmatDev);
}

static int matmat_check(const bemppcuda_matmat_args *a) {
    if (!a || !a->problems || a->nproblems <= 0) {
        bc_set_error("matmat: problem list missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->nrhs < 1 || a->nrhs > 8) {
        bc_set_error("matmat: nrhs must be 1..8 (got %d)", a->nrhs);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (!a->workspace || a->workspace_bytes < bemppcuda_matmat_workspace_bytes(a->nproblems)) {
        bc_set_error("matmat: workspace too small");
        return BEMPPCUDA_ERR_WORKSPACE;
    }
    for (int i = 0; i < a->nproblems; ++i) {
        const bemppcuda_matmat_problem &p = a->problems[i];
        if (!p.a || !p.x || !p.y || p.rows <= 0 || p.cols <= 0 || p.lda < p.cols || p.ldx < a->nrhs ||
            p.ldy < a->nrhs) {
            bc_set_error("matmat: problem %d has missing pointers or inconsistent sizes / strides", i);
            return BEMPPCUDA_ERR_INVALID;
        }
        if ((reinterpret_cast<uintptr_t>(p.a) | reinterpret_cast<uintptr_t>(p.x) |
             reinterpret_cast<uintptr_t>(p.y)) % 16 != 0) {
            bc_set_error("matmat: problem %d: complex128 arrays must be 16-byte aligned", i);
            return BEMPPCUDA_ERR_INVALID;
        }
    }
    return BEMPPCUDA_OK;
}

extern "C" int bemppcuda_matmat_prepare(bemppcuda_matmat_args *a, void *stream) {
    int rc = matmat_check(a);
    if (rc) return rc;
    MatmatDev *host = new MatmatDev[a->nproblems];
    int64_t blocks = 0;
    for (int i = 0; i < a->nproblems; ++i) {
        const bemppcuda_matmat_problem &p = a->problems[i];
        MatmatDev &d = host[i];
        d.a = static_cast<const double2 *>(p.a);
        d.x = static_cast<const double2 *>(p.x);
        d.y = static_cast<double2 *>(p.y);
        d.rows = p.rows;
        d.cols = p.cols;
        d.lda = p.lda;
        d.ldx = p.ldx;
        d.ldy = p.ldy;
        d.block_begin = blocks;
        blocks += (p.rows + MM_ROWS - 1) / MM_ROWS;
    }
    cudaError_t err = blocks > 0x7fffffffLL ? cudaErrorInvalidValue
                                            : cudaMemcpyAsync(a->workspace, host, sizeof(MatmatDev) * a->nproblems,
                                                              cudaMemcpyHostToDevice, (cudaStream_t)stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize((cudaStream_t)stream);
    delete[] host;
    if (err != cudaSuccess) {
        bc_set_error("matmat_prepare: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    a->blocks = blocks;
    return BEMPPCUDA_OK;
}

extern "C" int bemppcuda_matmat_launch(const bemppcuda_matmat_args *a, void *stream) {
    if (!a || !a->workspace || a->nproblems <= 0 || a->blocks <= 0 || a->nrhs < 1 || a->nrhs > 8) {
        bc_set_error("matmat_launch: call bemppcuda_matmat_prepare first");
        return BEMPPCUDA_ERR_INVALID;
    }
    const MatmatDev *probs = static_cast<const MatmatDev *>(a->workspace);
    cudaError_t err = cudaSuccess;
    switch (a->nrhs) {
    case 1: err = launch_matmat<1>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 2: err = launch_matmat<2>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 3: err = launch_matmat<3>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 4: err = launch_matmat<4>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 5: err = launch_matmat<5>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 6: err = launch_matmat<6>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    case 7: err = launch_matmat<7>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    default: err = launch_matmat<8>(probs, a->nproblems, a->blocks, (cudaStream_t)stream); break;
    }
    if (err != cudaSuccess) {
        bc_set_error("matmat_launch: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
