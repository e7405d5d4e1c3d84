// Batched multi-right-hand-side products Y_p = A_p X_p of dense complex128
// operators: the device counterpart of DenseDiscreteBoundaryOperator._matmat
// (api/assembly/discrete_boundary_operator.py:192-198, ndarray.dot on the
// host) for a list of operators with up to 8 right-hand sides each, in one
// launch; and the one-right-hand-side product of the solves (bemppcuda_gemv).
//
// With 8 right-hand sides each 16-byte matrix entry meets 8 complex FMAs
// (64 flops), so the product sits at the FP64 ridge of a B200 (4 flop / byte
// at HBM bandwidth is ~26 TFLOP/s, the FP64 pipe ~36).  2 to 8 right-hand
// sides run on the FP64 tensor cores (matmat_c128_tc below), which take the
// multiply-adds off the FP64 pipe and out of the issue slots, so the kernel
// is left to stream A.  One right-hand side of the batched call keeps the
// FP64-pipe kernel matmat_c128: a CTA of 8 warps owns 16 rows of one problem
// (2 rows per warp); columns go in tiles of 64.  A three-stage pipeline of
// asynchronous 16-byte copies (cp.async, L2 only) brings each tile of A
// (16 x 64, 16 KB) and the matching rows of X (transposed to xs[c][j], one
// padding element per row so the transposing stores spread over the banks)
// into shared memory two tiles ahead, about 32 KB in flight per CTA.  Each
// lane reads A(r, j) for its 2 rows and j = lane + 32 m, and every X(j, c)
// once for both rows; one barrier per tile.  Partial sums are reduced across
// the warp with shuffles at the end.  In both kernels a CTA's problem is
// found by binary search over the problems' first row blocks.
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
    int64_t wide;  // every row of A starts on a 32-byte boundary (A 32-byte aligned, lda even)
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

// ---------------------------------------------------------------------------------------------
// FP64 tensor cores (mma.sync m8n8k4 .f64; Blackwell's tcgen05 has no FP64 form).  The complex
// product is one real GEMM: a row of A read as its interleaved (re, im) doubles is a real row of
// length 2K, and X becomes the real 2K x 2N matrix B with, for complex column j of A and column c
// of X,
//   B[2j][2c] = Re X[j][c],   B[2j][2c+1] = Im X[j][c],
//   B[2j+1][2c] = -Im X[j][c], B[2j+1][2c+1] = Re X[j][c],
// so that (A B)[r][2c] = Re Y[r][c] and (A B)[r][2c+1] = Im Y[r][c].  A warp owns MT tiles of 8
// rows; per group of 4 complex columns lane (g, t) = (lane / 4, lane % 4) loads A[row g][j0 + t]
// as one 16-byte (re, im) pair straight from global memory (8 rows x 64 contiguous bytes per warp
// load, streamed past L1) and uses re as its A fragment of one k4 step and im as that of a second,
// the k index of both steps being t (the sum over k may be taken in any order, B follows it).  The
// B fragments (B[k = t][n = g]) come from X[j0 + t][c] with c = g / 2 (output columns 0-7 =
// complex columns 0-3) and 4 + g / 2 (columns 4-7, when NR > 4), cached in L1 since every warp of
// the problem reads the same X.  The accumulator fragment of lane (g, t), C[g][2t], C[g][2t + 1],
// is the complex entry Y[row g][4 n + t]: stored directly.  Columns beyond NR read zero.  Where
// the rows of A are 32-byte aligned a lane loads two consecutive complex entries at once
// (tc_group_wide) and runs the two k4 steps of both columns.
//
// From 5 right-hand sides on, the real form above takes 4 m8n8k4 products per 8 rows and 4 complex
// columns (2 k steps x 2 n8 tiles), which at 8 right-hand sides keeps the DMMA pipe about 3/4 busy
// at the bandwidth the kernel streams A.  Those sizes use Gauss's three-multiplication form instead
// (Higham, "Stability of a method for multiplying complex matrices with three real
// multiplications", SIAM J. Matrix Anal. Appl. 13, 1992):
//   T1 = Re A Re X,  T2 = Im A Im X,  T3 = (Re A + Im A)(Re X + Im X),
//   Re Y = T1 - T2,  Im Y = T3 - T1 - T2,
// three n8 tiles with n = complex column g (B[k = t][n = g] = X[j0 + t][g]) and k the complex
// column t of A: 3 products instead of 4, two FP64 additions per loaded A and X value.  The error
// stays normwise of the order of the unit roundoff times |A| |X| (Higham's bound).  Lane (g, t)
// ends with T1..T3 at row g, complex columns 2t and 2t + 1.
constexpr int TC_WARPS = 4;

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

// A is read once: keep it out of L1 (X and the other operands use it)
__device__ __forceinline__ double2 ld_stream(const double2 *p) {
    double2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}

__device__ __forceinline__ float2 ld_stream(const float2 *p) {
    float2 v;
    asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0,%1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}

template <int NR, int MT>
struct TcLayout {
    static constexpr bool GAUSS = NR > 4;      // three-multiplication form
    static constexpr int NT = GAUSS ? 3 : 1;   // n8 accumulator tiles (T1..T3, or 2 NR real columns)
    static constexpr int ROWS = 8 * MT;        // rows per CTA: its warps split the columns
};

// A[row][j], A[row][j + 1] with one 32-byte load (p 32-byte aligned), with a hint to fetch the
// 256-byte L2 stretch around it
__device__ __forceinline__ void ld_wide(const double2 *p, double2 &lo, double2 &hi) {
    unsigned long long a, b, c, d;
    asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.b64 {%0,%1,%2,%3}, [%4];\n"
                 : "=l"(a), "=l"(b), "=l"(c), "=l"(d)
                 : "l"(p));
    lo = make_double2(__longlong_as_double(a), __longlong_as_double(b));
    hi = make_double2(__longlong_as_double(c), __longlong_as_double(d));
}

// The products of one k4 step: lane (g, t) holds av[m] = A[row g of tile m][j] (zero when !jok)
// and fetches the B fragments of column j itself.
template <int NR, int MT>
__device__ __forceinline__ void tc_column(const MatmatDev &P, const double2 (&av)[MT], int64_t j, bool jok, int g,
                                          double (&acc)[MT][TcLayout<NR, MT>::NT][2]) {
    if constexpr (TcLayout<NR, MT>::GAUSS) {
        const double2 xv = (jok && g < NR) ? __ldg(P.x + j * P.ldx + g) : make_double2(0.0, 0.0);
        const double xs = xv.x + xv.y;
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            dmma(acc[m][0], av[m].x, xv.x);
            dmma(acc[m][1], av[m].y, xv.y);
            dmma(acc[m][2], av[m].x + av[m].y, xs);
        }
    } else {
        const int c = g >> 1;
        const double2 xv = (jok && c < NR) ? __ldg(P.x + j * P.ldx + c) : make_double2(0.0, 0.0);
        const double bre = (g & 1) ? xv.y : xv.x;   // B[2j][g]
        const double bim = (g & 1) ? xv.x : -xv.y;  // B[2j + 1][g]
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            dmma(acc[m][0], av[m].x, bre);
            dmma(acc[m][0], av[m].y, bim);
        }
    }
}

// 4 columns per warp, lane (g, t) taking column j0 + t with one 16-byte load per row; MASK: columns
// past the end read zero
template <int NR, int MT, bool MASK>
__device__ __forceinline__ void tc_group(const MatmatDev &P, const double2 *const (&arow)[MT], int64_t j0, int g,
                                         int t, double (&acc)[MT][TcLayout<NR, MT>::NT][2]) {
    const int64_t j = j0 + t;
    const bool jok = !MASK || j < P.cols;
    double2 av[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) av[m] = jok ? ld_stream(arow[m] + j) : make_double2(0.0, 0.0);
    tc_column<NR, MT>(P, av, j, jok, g, acc);
}

// 8 columns per warp, lane (g, t) taking columns j0 + 2t and j0 + 2t + 1 with one 32-byte load per
// row (rows 32-byte aligned, j0 even, both columns in range): half the load instructions, and twice
// the bytes per request in flight
template <int NR, int MT>
__device__ __forceinline__ void tc_group_wide(const MatmatDev &P, const double2 *const (&arow)[MT], int64_t j0,
                                              int g, int t, double (&acc)[MT][TcLayout<NR, MT>::NT][2]) {
    const int64_t j = j0 + 2 * t;
    double2 lo[MT], hi[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) ld_wide(arow[m] + j, lo[m], hi[m]);
    tc_column<NR, MT>(P, lo, j, true, g, acc);
    tc_column<NR, MT>(P, hi, j + 1, true, g, acc);
}

// A CTA owns 8 MT rows of one problem; its TC_WARPS warps split the columns in steps of
// 16 TC_WARPS (warp w takes columns 16 w .. 16 w + 15 of each step, so a step reads one contiguous
// 256-byte-per-warp stretch of every row), then add their accumulators in shared memory in a fixed
// order.  Splitting the columns instead of the rows keeps four times as many CTAs for the same
// matrix (problems of a few thousand rows still fill the GPU) without atomics.  Problems whose rows
// start on 32-byte boundaries (MatmatDev::wide) stream A with 32-byte loads, the others with 16-byte
// loads; the ragged last columns always take the masked 16-byte form.
// Compiled for 7 CTAs per SM (72 registers, some spill to L1): the product waits on its loads, and
// 28 warps per SM keep more of them in flight than the 20 that 88 registers allowed.  25 x 8192^2
// x 8 right-hand sides, CUDA events: 4.77 TB/s (real form, 16-byte loads, 5 CTAs / SM), 5.3
// (8 CTAs / SM), 5.7 (three-multiplication form), 6.5 (32-byte loads), 6.7 (7 CTAs / SM; 6 and 8:
// 6.6 and 6.5).
#ifndef BC_MATMAT_TC_MIN_BLOCKS
#define BC_MATMAT_TC_MIN_BLOCKS 7
#endif

template <int NR, int MT>
__global__ void __launch_bounds__(TC_WARPS * 32, BC_MATMAT_TC_MIN_BLOCKS) matmat_c128_tc(const MatmatDev *__restrict__ probs,
                                                                                       int nproblems) {
    using L = TcLayout<NR, MT>;
    constexpr int GW = 4;                 // columns per group
    constexpr int STEP = 16 * TC_WARPS;  // columns per step of the CTA
    __shared__ double red[TC_WARPS - 1][MT][L::NT][2][32];
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
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int64_t r0 = (b - P.block_begin) * L::ROWS;  // < P.rows by construction of the blocks
    const double2 *arow[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) arow[m] = P.a + min(r0 + 8 * m + g, P.rows - 1) * P.lda;
    double acc[MT][L::NT][2];
#pragma unroll
    for (int m = 0; m < MT; ++m)
#pragma unroll
        for (int n = 0; n < L::NT; ++n) acc[m][n][0] = acc[m][n][1] = 0.0;
    const int64_t full = P.cols / STEP * STEP;
    if (P.wide) {
        for (int64_t j0 = 16 * warp; j0 < full; j0 += STEP) {
#pragma unroll
            for (int u = 0; u < 2; ++u) tc_group_wide<NR, MT>(P, arow, j0 + 8 * u, g, t, acc);
        }
    } else {
        for (int64_t j0 = 16 * warp; j0 < full; j0 += STEP) {
#pragma unroll
            for (int u = 0; u < 4; ++u) tc_group<NR, MT, false>(P, arow, j0 + u * GW, g, t, acc);
        }
    }
    for (int64_t j0 = full + 16 * warp; j0 < P.cols; j0 += STEP)
        for (int u = 0; u < 4 && j0 + u * GW < P.cols; ++u) tc_group<NR, MT, true>(P, arow, j0 + u * GW, g, t, acc);
    if (warp > 0) {
#pragma unroll
        for (int m = 0; m < MT; ++m)
#pragma unroll
            for (int n = 0; n < L::NT; ++n) {
                red[warp - 1][m][n][0][lane] = acc[m][n][0];
                red[warp - 1][m][n][1][lane] = acc[m][n][1];
            }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int w = 0; w < TC_WARPS - 1; ++w)
#pragma unroll
            for (int m = 0; m < MT; ++m)
#pragma unroll
                for (int n = 0; n < L::NT; ++n) {
                    acc[m][n][0] += red[w][m][n][0][lane];
                    acc[m][n][1] += red[w][m][n][1][lane];
                }
#pragma unroll
        for (int m = 0; m < MT; ++m) {
            const int64_t r = r0 + 8 * m + g;
            if constexpr (L::GAUSS) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int c = 2 * t + q;
                    const double t12 = acc[m][0][q] + acc[m][1][q];
                    if (r < P.rows && c < NR)
                        P.y[r * P.ldy + c] = make_double2(acc[m][0][q] - acc[m][1][q], acc[m][2][q] - t12);
                }
            } else {
#pragma unroll
                for (int n = 0; n < L::NT; ++n) {
                    const int c = 4 * n + t;
                    if (r < P.rows && c < NR) P.y[r * P.ldy + c] = make_double2(acc[m][n][0], acc[m][n][1]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// One right-hand side (the GMRES matvec): y = A x for a row-major complex matrix, HBM-bound.  The
// matrix is read like a copy reads its source: CTA b takes segment b % S of row b / S (S segments
// of GV_SEG entries per row), so consecutive CTAs stream consecutive memory; each thread loads
// GV_PER entries GV_THREADS apart (coalesced, all in flight at once, streamed past L1), multiplies
// by x (through L1), and the CTA's sum goes to y[row] with one atomic add per component, y having
// been zeroed.  Sums in the matrix's precision; the order of the atomic adds is not fixed.
template <typename C>
struct GemvTraits;
template <>
struct GemvTraits<double2> {
    using R = double;
};
template <>
struct GemvTraits<float2> {
    using R = float;
};

constexpr int GV_THREADS = 256;
constexpr int GV_PER = 8;  // 32 KB segments for complex128 (4 and 16 measured slower)
constexpr int64_t GV_SEG = (int64_t)GV_THREADS * GV_PER;

template <typename C>
__global__ void __launch_bounds__(GV_THREADS) gemv_segments(const C *__restrict__ a, int64_t cols, int64_t lda,
                                                             int64_t segs, int64_t block0, const C *__restrict__ x,
                                                             C *y) {
    using R = typename GemvTraits<C>::R;
    const int64_t blk = block0 + blockIdx.x;
    const int64_t row = blk / segs, j0 = (blk - row * segs) * GV_SEG + threadIdx.x;
    const C *ar = a + row * lda;
    C av[GV_PER], xv[GV_PER];
#pragma unroll
    for (int u = 0; u < GV_PER; ++u) {
        const int64_t j = j0 + (int64_t)u * GV_THREADS;
        if (j < cols) {
            av[u] = ld_stream(ar + j);
            xv[u] = __ldg(x + j);
        } else {
            av[u].x = av[u].y = xv[u].x = xv[u].y = 0;
        }
    }
    R sr = 0, si = 0;
#pragma unroll
    for (int u = 0; u < GV_PER; ++u) {
        sr = fma(av[u].x, xv[u].x, fma(-av[u].y, xv[u].y, sr));
        si = fma(av[u].x, xv[u].y, fma(av[u].y, xv[u].x, si));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, off);
        si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    __shared__ R part[2][GV_THREADS / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        part[0][warp] = sr;
        part[1][warp] = si;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        R tr = 0, ti = 0;
#pragma unroll
        for (int w = 0; w < GV_THREADS / 32; ++w) {
            tr += part[0][w];
            ti += part[1][w];
        }
        atomicAdd(&y[row].x, tr);
        atomicAdd(&y[row].y, ti);
    }
}

}  // namespace bc

using namespace bc;

// m8 tiles per warp (rows per CTA = 8 x this): 2 measured fastest against 4 on 25 x 8192^2, 64 x
// 2048^2, 3 x 8192^2 and 1 x 4096^2 with eight right-hand sides
#ifndef BC_MATMAT_TC_MT
#define BC_MATMAT_TC_MT 2
#endif

// rows per CTA of the kernel that serves nrhs right-hand sides: tensor cores from 2 up
static int64_t matmat_rows_per_block(int nrhs) {
    return nrhs >= 2 ? (int64_t)8 * BC_MATMAT_TC_MT : (int64_t)MM_ROWS;
}

template <int NR>
static cudaError_t launch_matmat_tc(const MatmatDev *probs, int nproblems, int64_t blocks, cudaStream_t st) {
    matmat_c128_tc<NR, BC_MATMAT_TC_MT><<<dim3((unsigned)blocks), TC_WARPS * 32, 0, st>>>(probs, nproblems);
    return cudaGetLastError();
}

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
        d.wide = (reinterpret_cast<uintptr_t>(p.a) % 32 == 0 && p.lda % 2 == 0) ? 1 : 0;
        const int64_t rpb = matmat_rows_per_block(a->nrhs);
        blocks += (p.rows + rpb - 1) / rpb;
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
    const cudaStream_t st = (cudaStream_t)stream;
    switch (a->nrhs) {
    case 1: err = launch_matmat<1>(probs, a->nproblems, a->blocks, st); break;
    case 2: err = launch_matmat_tc<2>(probs, a->nproblems, a->blocks, st); break;
    case 3: err = launch_matmat_tc<3>(probs, a->nproblems, a->blocks, st); break;
    case 4: err = launch_matmat_tc<4>(probs, a->nproblems, a->blocks, st); break;
    case 5: err = launch_matmat_tc<5>(probs, a->nproblems, a->blocks, st); break;
    case 6: err = launch_matmat_tc<6>(probs, a->nproblems, a->blocks, st); break;
    case 7: err = launch_matmat_tc<7>(probs, a->nproblems, a->blocks, st); break;
    default: err = launch_matmat_tc<8>(probs, a->nproblems, a->blocks, st); break;
    }
    if (err != cudaSuccess) {
        bc_set_error("matmat_launch: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}

extern "C" int bemppcuda_gemv(const void *a, int64_t rows, int64_t cols, int64_t lda, const void *x, void *y,
                              int32_t complex64, void *stream) {
    if (rows < 0 || cols < 0 || lda < cols || ((rows > 0 && cols > 0) && (!a || !x)) || (rows > 0 && !y)) {
        bc_set_error("gemv: missing pointers or inconsistent sizes (rows %lld, cols %lld, lda %lld)",
                     (long long)rows, (long long)cols, (long long)lda);
        return BEMPPCUDA_ERR_INVALID;
    }
    const size_t elem = complex64 ? 8 : 16;
    if ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) % elem) {
        bc_set_error("gemv: arrays must be aligned to their element size");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (rows == 0) return BEMPPCUDA_OK;
    const cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(y, 0, (size_t)rows * elem, st);
    if (err != cudaSuccess) {
        bc_set_error("gemv: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    if (cols == 0) return BEMPPCUDA_OK;
    const int64_t segs = (cols + GV_SEG - 1) / GV_SEG;
    const int64_t total = rows * segs;
    constexpr int64_t kMaxGrid = 0x7fffffffLL;
    for (int64_t b0 = 0; b0 < total; b0 += kMaxGrid) {
        const unsigned n = (unsigned)min(total - b0, kMaxGrid);
        if (complex64)
            gemv_segments<float2><<<n, GV_THREADS, 0, st>>>(static_cast<const float2 *>(a), cols, lda, segs, b0,
                                                            static_cast<const float2 *>(x), static_cast<float2 *>(y));
        else
            gemv_segments<double2><<<n, GV_THREADS, 0, st>>>(static_cast<const double2 *>(a), cols, lda, segs, b0,
                                                             static_cast<const double2 *>(x),
                                                             static_cast<double2 *>(y));
    }
    return bc_check_launch("gemv");
}
