/*
 * bemppcuda: B200 (sm_100a) dense Galerkin assembly and potential evaluation.
 *
 * Flat C ABI.  Every data pointer is a DEVICE pointer unless the field says
 * HOST; the library never allocates, frees or retains caller memory.  Every
 * entry point returns 0 on success or a negative status and never aborts;
 * bemppcuda_last_error() gives the message of the last failure on the
 * calling thread.  Work is enqueued on the given CUDA stream (NULL = legacy
 * default stream) and is asynchronous with respect to the host.
 *
 * The entry points replace the device back ends that bempp-cl selects
 * through bempp_cl/core/dispatcher.py:
 *   bemppcuda_assemble_regular   <- numba_assemblers.dense_assembler
 *                                   (bempp_cl/core/numba_assemblers.py:58-112)
 *   bemppcuda_assemble_singular  <- numba_assemblers.singular_assembler
 *                                   (bempp_cl/core/numba_assemblers.py:6-55)
 *   bemppcuda_evaluate_potential <- numba_assemblers.potential_assembler
 *                                   evaluator (bempp_cl/core/numba_assemblers.py:115-164)
 *   bemppcuda_grid_geometry      <- Grid._compute_geometric_quantities
 *                                   (bempp_cl/api/grid/grid.py:552-590)
 */
#ifndef BEMPPCUDA_H
#define BEMPPCUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define BEMPPCUDA_OK 0
#define BEMPPCUDA_ERR_INVALID (-1)     /* bad argument: size, pointer, id */
#define BEMPPCUDA_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define BEMPPCUDA_ERR_UNSUPPORTED (-3) /* valid request this build does not implement */
#define BEMPPCUDA_ERR_WORKSPACE (-4)   /* workspace smaller than required */

/* Green's functions (kernel_type strings of bempp_cl/core/numba_kernels.py:39-64) */
#define BEMPPCUDA_LAPLACE_SLP 0
#define BEMPPCUDA_LAPLACE_DLP 1
#define BEMPPCUDA_LAPLACE_ADLP 2
#define BEMPPCUDA_HELMHOLTZ_SLP 3
#define BEMPPCUDA_HELMHOLTZ_DLP 4
#define BEMPPCUDA_HELMHOLTZ_ADLP 5
#define BEMPPCUDA_MODHELM_SLP 6
#define BEMPPCUDA_MODHELM_DLP 7
#define BEMPPCUDA_MODHELM_ADLP 8
#define BEMPPCUDA_FARFIELD_SLP 9
#define BEMPPCUDA_FARFIELD_DLP 10
/* Fused Helmholtz combined field: DLP + eta * SLP with params = (Re k, Im k,
   Re eta, Im eta).  No reference counterpart as one kernel: the reference
   assembles the two operators separately and adds the weak forms
   (boundary_operator.py:134-169); this computes the same sum in one pass. */
#define BEMPPCUDA_HELMHOLTZ_COMBINED 11

/* assembly types (assembly_type strings of numba_kernels.py:11-34) */
#define BEMPPCUDA_ASM_SCALAR 0      /* default_scalar */
#define BEMPPCUDA_ASM_LAPLACE_HYP 1 /* laplace_hypersingular */
#define BEMPPCUDA_ASM_HELM_HYP 2    /* helmholtz_hypersingular */
#define BEMPPCUDA_ASM_MODHELM_HYP 3 /* modified_helmholtz_hypersingular */
#define BEMPPCUDA_ASM_EFIE 4        /* maxwell_electric_field (+ _far_field for potentials) */
#define BEMPPCUDA_ASM_MFIE 5        /* maxwell_magnetic_field (+ _far_field for potentials) */

/* shape sets */
#define BEMPPCUDA_SHAPE_P0 0  /* p0_discontinuous, 1 function */
#define BEMPPCUDA_SHAPE_P1 1  /* p1_discontinuous, 3 functions */
#define BEMPPCUDA_SHAPE_RWG 2 /* rwg0 / snc0 reference functions, Piola-mapped */

/* precision of the regular (non-adjacent) element pairs */
#define BEMPPCUDA_FP64 0
#define BEMPPCUDA_MIXED 1 /* FP32 kernel evaluation, FP64 per-entry accumulation */

/* geometry record: BEMPPCUDA_GEOM_FIELDS doubles per element, stored field-major
   (field f of element e at geom[f * nelements + e]):
   0-2 vertex 0, 3-5 v1 - v0, 6-8 v2 - v0, 9-11 unit normal, 12 integration
   element, 13-15 edge lengths |v0-v1|, |v2-v0|, |v1-v2|, 16-21 J (J^T J)^-1
   row-major (3 x 2), 22-24 centroid. */
#define BEMPPCUDA_GEOM_FIELDS 25

#define BEMPPCUDA_MAX_REGULAR_POINTS 16

/* One function space restricted to its support elements. */
typedef struct {
    int32_t shapeset;           /* BEMPPCUDA_SHAPE_* */
    int32_t nshape;             /* 1 or 3 */
    int64_t nsupport;           /* number of support elements */
    const uint32_t *support;    /* (nsupport,) element ids, increasing */
    const uint32_t *l2g;        /* (nelements, nshape) global dof of each local function */
    const double *mult;         /* (nelements, nshape) local multipliers */
    const int32_t *normal_mult; /* (nelements,) +1/-1; NULL means all +1 */
    int64_t ndofs;              /* global dof count (matrix extent) */
    int32_t dof_is_position;    /* 1: nshape == 1, dof of support[i] is i, mult 1 */
    int32_t pad;
} bemppcuda_space;

typedef struct {
    int64_t nvertices;
    int64_t nelements;
    const double *geom;      /* BEMPPCUDA_GEOM_FIELDS * nelements, from bemppcuda_grid_geometry */
    const int32_t *elements; /* (nelements, 3) vertex ids, element-major */
} bemppcuda_grid;

/* Regular-pair assembly: result[l2g_test, l2g_trial] (+)= sum over element pairs
   that share no vertex when the grids are identical (numba_kernels.py:980-2278). */
typedef struct {
    int32_t kernel;     /* BEMPPCUDA_* Green's function */
    int32_t assembly;   /* BEMPPCUDA_ASM_* */
    int32_t precision;  /* BEMPPCUDA_FP64 or BEMPPCUDA_MIXED: DP0 scalar kernels; P1 single, double,
                           adjoint double layer and hypersingular (Helmholtz with Re k > 0, Laplace,
                           modified Helmholtz), P1 beside P0 for the scalar operators; Maxwell electric and magnetic fields (Re k > 0);
                           6-point rule.
                           Other operators return BEMPPCUDA_ERR_UNSUPPORTED under MIXED */
    int32_t is_complex; /* result is complex128 (1) or float64 (0) */
    double params[4];   /* kernel parameters: (Re k, Im k) or (omega) */
    bemppcuda_grid test_grid;
    bemppcuda_grid trial_grid;
    bemppcuda_space test;  /* dual_to_range */
    bemppcuda_space trial; /* domain */
    int32_t grids_identical;
    int32_t nq;                 /* regular rule size <= BEMPPCUDA_MAX_REGULAR_POINTS */
    const double *quad_points;  /* HOST (nq, 2) reference points */
    const double *quad_weights; /* HOST (nq,) */
    void *result;               /* (rows, ld) row-major float64 or complex128 */
    int64_t ld;                 /* row stride in entries */
    int32_t overwrite;          /* DP0 fast path only: store instead of add, zero for adjacent pairs */
    int32_t no_symmetry;        /* 0: when test and trial are the same space of one grid (same support, dof
                                   map, multiplier, normal-multiplier and geometry pointers; DP0, P1 / DP1 /
                                   P0, RWG with SNC) and k is real, one sweep over the pairs i < j gives
                                   A_ij and A_ji; 1: always evaluate every entry separately */
    double phase_radius;        /* R_test + R_trial, R = largest centroid-to-vertex distance of a grid;
                                   lets the mixed path skip the phase range reduction when
                                   |k| * phase_radius <= 1; 0 = unknown (always reduce) */
    int64_t row_begin;          /* symmetric sweep only: evaluate the pairs (i, j), i <= j, with rows i in */
    int64_t row_end;            /* [row_begin, row_end) (writing A_ij and A_ji); 0, 0 = all rows.  Rows of
                                   block [b, e) are complete once the blocks before it and this call ran */
    int32_t result_is_zero;     /* 1: the caller guarantees that result holds zeros.  Symmetric P1 / P0
                                   single-layer and hypersingular sweeps then store only the blocks of
                                   the pairs i < j and form A = U + U^T in one pass over the matrix,
                                   half the global atomics; 0: accumulate both blocks into result */
    int32_t pad2;
    void *tresult;              /* NULL, or with row_begin / row_end (the DP0 symmetric sweep): a stripe
                                   of the upper triangle into two local buffers of the same layout,
                                   A_ij at result[(i - row_begin) * ld + (j - col_begin)] and the
                                   transposed entry A_ji at tresult[(i - row_begin) * ld + (j - col_begin)],
                                   for the swept pairs i <= j (entries with j < i are not written);
                                   Helmholtz single / double / adjoint double layer, combined field and
                                   Laplace single layer (others: BEMPPCUDA_ERR_UNSUPPORTED) */
    int64_t col_begin;          /* first column held by result / tresult (<= row_begin) */
} bemppcuda_regular_args;

/* Singular pairs (Sauter-Schwab), the arrays of
   _SingularQuadratureRuleInterfaceGalerkin.get_arrays (core/singular_assembler.py:251-278). */
typedef struct {
    int32_t kernel;
    int32_t assembly;
    int32_t is_complex;
    int32_t pad0;
    double params[4];
    bemppcuda_grid grid;
    bemppcuda_space test;
    bemppcuda_space trial;
    int64_t npairs;
    int64_t npoints_table;        /* columns of the point tables */
    const double *test_points;    /* (npoints_table, 2) point-major */
    const double *trial_points;   /* (npoints_table, 2) */
    const double *weights;        /* weight table */
    int64_t nweights;
    const uint32_t *test_elements;
    const uint32_t *trial_elements;
    const uint32_t *test_offsets;
    const uint32_t *trial_offsets;
    const uint32_t *weights_offsets;
    const uint32_t *npoints;
    /* output: exactly one of the two */
    void *values;      /* flat (npairs, nshape_test, nshape_trial), accumulated into */
    void *dense;       /* or: scatter value * multipliers into result[l2g_test, l2g_trial] */
    int64_t ld;        /* row stride of dense */
    double diag_shift; /* added to the coincident entries of a DP0 dense output, times the
                          integration element / 2 (the -1/2 I term of a combined-field form) */
    double phase_radius; /* 2 x largest centroid-to-vertex distance of the grid, or 0 (unknown):
                            when |k| * phase_radius <= 1 the DP0 path factors exp(ikr) about the
                            centroid distance (|r - r_c| <= R_i + R_j holds for adjacent pairs too) */
    int64_t mirror_weights_offset; /* dense output with the same space on both sides and every pair
                                      listed in both orders: the pairs whose weights start at this offset
                                      use a rule that is symmetric under exchanging test and trial points
                                      (the vertex-adjacent rule), so the pair with test < trial adds both
                                      entries (blocks) and its reverse adds nothing -- DP0 scalar kernels,
                                      and on P1 x P1 the single layers and hypersingular operators; 0 = off */
} bemppcuda_singular_args;

/* Potential / far-field evaluation (numba_kernels.py:1788-1849, 2281-2570). */
typedef struct {
    int32_t kernel;   /* Green's function; far-field kernels treat points as directions */
    int32_t assembly; /* BEMPPCUDA_ASM_SCALAR, _EFIE or _MFIE */
    int32_t precision; /* BEMPPCUDA_FP64, or BEMPPCUDA_MIXED (FP32 point-source pairs, FP64 per-element
                          phase, amplitude and sums) for Laplace, Helmholtz (Re k > 0, real or complex k)
                          and modified Helmholtz (omega > 0) single / double layer potentials,
                          Helmholtz far fields and the Maxwell magnetic potential and far field
                          (Re k > 0); other kernels return BEMPPCUDA_ERR_UNSUPPORTED under MIXED */
    int32_t pad0;
    double params[4];
    bemppcuda_grid grid;
    bemppcuda_space space;      /* nshape and shapeset; l2g / mult unused */
    int32_t nq;
    int32_t pad1;
    const double *quad_points;  /* HOST (nq, 2) */
    const double *quad_weights; /* HOST (nq,) */
    int64_t npoints;
    const double *points;       /* (npoints, 3) point-major */
    const double *coefficients; /* complex128 (nelements * nshape): element-local coefficients */
    void *result;               /* complex128 (kdim, npoints) */
    void *workspace;            /* bemppcuda_potential_workspace_bytes() bytes */
    int64_t workspace_bytes;
    double phase_radius;  /* largest centroid-to-vertex distance R of the source grid, or 0 (unknown):
                             scalar potentials with a real wavenumber factor exp(ikr) about each
                             element's centroid and skip the range reduction when |k| R <= 1.
                             Required (> 0) under BEMPPCUDA_MIXED, which evaluates an element's
                             sources in FP64 for points within 4 k R of its centroid (FP32 r^2 of a
                             point next to the surface would lose accuracy); BEMPPCUDA_ERR_INVALID
                             otherwise */
} bemppcuda_potential_args;

/* Batched DP0 assembly (many grids / wavenumbers in one persistent launch).
   No single reference counterpart: the reference assembles one operator per
   weak_form() call (core/dense_assembler.py:49-98); this assembles a list of
   them.  Each problem has identical full-support DP0 test and trial spaces on
   its own grid (rows = columns = elements). */
typedef struct {
    bemppcuda_grid grid;
    const uint32_t *support; /* (nelements,) 0, 1, ..., nelements - 1 */
    void *result;            /* complex128 (nelements, ld), every entry written */
    int64_t ld;
    double params[4];        /* (Re k, Im k, Re eta, Im eta) */
    double phase_radius;     /* 2 x largest centroid-to-vertex distance of the grid (0 = unknown) */
    int32_t precision;       /* BEMPPCUDA_FP64 or BEMPPCUDA_MIXED */
    int32_t pad;
    int64_t pair_begin;      /* first singular pair of this problem in the concatenated arrays */
    int64_t pair_count;
} bemppcuda_batch_problem;

typedef struct {
    int32_t kernel;                           /* BEMPPCUDA_HELMHOLTZ_SLP or _COMBINED, for all problems */
    int32_t nproblems;
    const bemppcuda_batch_problem *problems;  /* HOST array of nproblems entries */
    int32_t nq;                               /* must be 6 */
    int32_t blocks_per_sm;                    /* persistent grid = blocks_per_sm x SMs (0: 4) */
    const double *quad_points;                /* HOST (nq, 2) */
    const double *quad_weights;               /* HOST (nq,) */
    int64_t npairs;                           /* singular pairs of all problems, concatenated */
    const double *test_points;                /* shared Sauter-Schwab tables (P, 2) */
    const double *trial_points;
    const double *weights;
    const uint32_t *test_elements;            /* element ids local to each problem's grid */
    const uint32_t *trial_elements;
    const uint32_t *test_offsets;
    const uint32_t *trial_offsets;
    const uint32_t *weights_offsets;
    const uint32_t *npoints;
    double diag_shift;                        /* + diag_shift * area on coincident entries */
    int32_t rows_per_item;                    /* test elements per work item, 1..32 (0: 32) */
    int32_t pad;
    void *workspace;                          /* bemppcuda_batch_workspace_bytes(nproblems) bytes */
    int64_t workspace_bytes;
} bemppcuda_batch_args;

/* L2 identity (mass matrix) of two spaces on one grid as COO triplets.
   Replaces l2_identity_kernel (core/numba_kernels.py:713-769) with
   default_sparse_kernel (:935-976) and the triplet assembly of
   SparseAssembler.assemble (core/sparse_assembler.py:17-70): for every
   element e of `elements` (the elements in both supports) and local
   functions i (test), j (trial), entry e * nt * ns + i * ns + j holds
       row = test.l2g[e, i], col = trial.l2g[e, j],
       value = test.mult[e, i] * trial.mult[e, j] * |J_e| * sum_q w_q phi_i(q) . psi_j(q).
   Repeated (row, col) pairs are to be summed by the caller (as coo -> csr). */
#define BEMPPCUDA_BASIS_SCALAR 0 /* P0 / P1 / DP1 values */
#define BEMPPCUDA_BASIS_RWG 1    /* l_i / |J| J r_i (maxwell_spaces.py:678-712) */
#define BEMPPCUDA_BASIS_SNC 2    /* n x the RWG value, n times the normal multiplier (:716-757) */

typedef struct {
    bemppcuda_grid grid;
    bemppcuda_space test;       /* dual_to_range */
    bemppcuda_space trial;      /* domain */
    int32_t test_kind;          /* BEMPPCUDA_BASIS_*: both scalar, or both RWG / SNC */
    int32_t trial_kind;
    int64_t nelements;
    const uint32_t *elements;   /* (nelements,) device, elements in both supports */
    int32_t nq;                 /* rule size <= BEMPPCUDA_MAX_REGULAR_POINTS */
    int32_t pad;
    const double *quad_points;  /* HOST (nq, 2) */
    const double *quad_weights; /* HOST (nq,) */
    int64_t *rows;              /* device outputs, nelements * nt * ns entries each */
    int64_t *cols;
    double *values;
} bemppcuda_identity_args;

/* Batched multi-right-hand-side products Y_p = A_p X_p of dense complex128
   operators (interleaved re / im, row-major), one launch for the whole list.
   Replaces DenseDiscreteBoundaryOperator._matmat
   (api/assembly/discrete_boundary_operator.py:192-198, a host ndarray.dot per
   operator) for operators that stay on the device. */
typedef struct {
    const void *a;  /* complex128 (rows, cols), row stride lda elements; 16-byte aligned */
    const void *x;  /* complex128 (cols, nrhs), row stride ldx */
    void *y;        /* complex128 (rows, nrhs), row stride ldy; overwritten */
    int64_t rows, cols, lda, ldx, ldy;
} bemppcuda_matmat_problem;

typedef struct {
    int32_t nproblems;
    int32_t nrhs;                             /* 1..8, the same for every problem */
    const bemppcuda_matmat_problem *problems; /* HOST array of nproblems entries */
    void *workspace;                          /* bemppcuda_matmat_workspace_bytes(nproblems) bytes */
    int64_t workspace_bytes;
    int64_t blocks;                           /* written by bemppcuda_matmat_prepare */
} bemppcuda_matmat_args;

int bemppcuda_version(void);
int bemppcuda_last_error(char *buffer, int64_t length);

/* Per-element geometry from vertices (3, nv) vertex-major xyz and elements
   (nelements, 3).  Writes BEMPPCUDA_GEOM_FIELDS * nelements doubles. */
int bemppcuda_grid_geometry(const double *vertices, int64_t nvertices, const int32_t *elements, int64_t nelements,
                            double *geom, void *stream);

int bemppcuda_assemble_regular(const bemppcuda_regular_args *args, void *stream);
int bemppcuda_assemble_singular(const bemppcuda_singular_args *args, void *stream);

/* Matrix-free FP64 apply of the regular part: y += A_reg x, complex128 vectors (x: trial.nsupport
   entries, y: test.nsupport), A_reg the Galerkin matrix of the non-adjacent element pairs evaluated on
   the fly (never stored).  Adjacent pairs and the diagonal contribute nothing here: they are the
   singular part.  Replaces the residual product of the reference's solve, b - A x with the assembled
   weak form (api/linalg/iterative_solvers.py:47-93, discrete_boundary_operator.py:192-198), for a
   matrix that is held in lower precision: same regular entries as bemppcuda_assemble_regular in
   FP64, summed in another order.  Scope: Laplace / Helmholtz single, double, adjoint double layer
   and the combined field (params as for the assembly) on one DP0 space of one grid (identity dof
   map, the same device arrays on both sides) with the 6-point rule and precision FP64; anything else
   returns BEMPPCUDA_ERR_UNSUPPORTED.  result / ld / overwrite / row_begin / row_end are ignored.
   y is updated with atomics: the summation order is not deterministic. */
int bemppcuda_apply_regular(const bemppcuda_regular_args *args, const void *x, void *y, void *stream);

/* Projections of a function onto a scalar space (P0 / P1 shapesets): the vectorized projection of
   GridFunction (api/assembly/grid_function.py, _project_function_vectorized), on the device.
   bemppcuda_quadrature_points writes the global points and the unit normals (times the normal
   multipliers) of every (support element, point) of the nq-point rule, in the reference's
   vectorized-callable layout: points / normals (3, nsupport * nq), component-major, point index
   k * nq + q for support element k; normals may be NULL.  The caller evaluates its function there
   (on the device or the host) and passes the complex128 values (nsupport * nq);
   bemppcuda_project zeroes out (ndofs complex128) and adds
   mult(e, i) |J_e| sum_q w_q phi_i(q) f(e, q) at l2g(e, i) with FP64 atomics (order not fixed). */
int bemppcuda_quadrature_points(const bemppcuda_grid *grid, const bemppcuda_space *space, int32_t nq,
                                const double *quad_points, const double *quad_weights, double *points,
                                double *normals, void *stream);
int bemppcuda_project(const bemppcuda_grid *grid, const bemppcuda_space *space, int32_t nq,
                      const double *quad_points, const double *quad_weights, const void *values, void *out,
                      void *stream);

/* Bytes of the source table (0 for no sources; -1 when the size overflows int64, which
   bemppcuda_evaluate_potential rejects with BEMPPCUDA_ERR_INVALID). */
int64_t bemppcuda_potential_workspace_bytes(const bemppcuda_potential_args *args);
int bemppcuda_evaluate_potential(const bemppcuda_potential_args *args, void *stream);

/* Potential evaluation for callers that cannot allocate device memory.  No
   counterpart in the reference (its evaluator allocates host arrays freely).
   Same arguments and results as bemppcuda_evaluate_potential, but
   args->workspace / workspace_bytes are ignored: the source table goes into a
   fixed array of BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES doubles (24 MiB) that the
   library keeps on every GPU that loads it, so the call allocates nothing.
   It is meant for code that only receives input and output device buffers
   from a host application owning all device memory (a plugin inside a
   solver's memory pool, an embedding runtime without a CUDA allocation
   binding), where cudaMalloc may fail or would synchronize the device.
   Problems whose table exceeds the array (space.nsupport * nq * 14 doubles)
   are rejected with BEMPPCUDA_ERR_WORKSPACE.  All calls on a device share
   the array: calls that can overlap on the GPU race, so order them on one
   stream.  Every call made outside a stream capture looks the array's device
   address up again (it moves when the context is recreated, e.g. after
   cudaDeviceReset); a captured call reuses the last looked-up address, so
   make one call on a device before any stream capture starts there. */
#define BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES (3 * 1024 * 1024)
int bemppcuda_evaluate_potential_noalloc(const bemppcuda_potential_args *args, void *stream);

int64_t bemppcuda_batch_workspace_bytes(int32_t nproblems);
/* Upload the problem table into the workspace (host-to-device copy on the
   stream, then a stream synchronize); call again whenever the list changes. */
int bemppcuda_batch_prepare(const bemppcuda_batch_args *args, void *stream);
/* Reset the work counter, run the persistent regular-pair kernel over every
   (problem, tile) item and the batched singular kernel.  Device work only
   (a memset and two launches), so it can be captured in a CUDA graph once
   bemppcuda_batch_prepare has run. */
int bemppcuda_batch_launch(const bemppcuda_batch_args *args, void *stream);

int bemppcuda_assemble_identity(const bemppcuda_identity_args *args, void *stream);

int64_t bemppcuda_matmat_workspace_bytes(int32_t nproblems);
/* Check the list, upload it into the workspace (host-to-device copy, then a
   stream synchronize) and set args->blocks; call again whenever it changes. */
int bemppcuda_matmat_prepare(bemppcuda_matmat_args *args, void *stream);
/* One kernel launch over every problem's rows (device work only, so it can be
   captured in a CUDA graph once bemppcuda_matmat_prepare has run).  FP64
   sums; the order differs from a BLAS product's, so results agree with it to
   rounding, not bit for bit.  2 to 8 right-hand sides run on the FP64 tensor
   cores (mma.sync m8n8k4 .f64), 1 on the FP64 pipe; 5 to 8 use Gauss's
   three-multiplication complex product, whose error is bounded normwise
   (of the order of the unit roundoff times |A| |X|), so an imaginary part
   much smaller than that product may carry a larger relative error.
   Problems whose a is 32-byte aligned with an even lda are read with
   32-byte loads (faster); any 16-byte aligned layout is accepted. */
int bemppcuda_matmat_launch(const bemppcuda_matmat_args *args, void *stream);

/* y = A x, one right-hand side: the matvec of the solve (DenseDiscreteBoundaryOperator._matvec,
   api/assembly/discrete_boundary_operator.py:192-198, ndarray.dot on the host; scipy's GMRES calls
   it once per iteration, api/linalg/iterative_solvers.py:47-93).  A row-major (rows, cols) with row
   stride lda >= cols, x (cols,), y (rows,), all device arrays of complex128 (complex64 = 0) or
   complex64 (complex64 = 1), aligned to their element size.  HBM-bound stream of A; y is zeroed
   and receives the sums of row segments with atomic adds, in the matrix's precision: equal to a
   BLAS GEMV to rounding, not bit for bit, and not bit-reproducible from call to call. */
int bemppcuda_gemv(const void *a, int64_t rows, int64_t cols, int64_t lda, const void *x, void *y, int32_t complex64,
                   void *stream);

/* Measurement utility, no reference counterpart: launches `blocks` x 256
   threads that each run 32 independent FMAs per iteration in FP64
   (precision = BEMPPCUDA_FP64) or FP32 (otherwise); *flops receives the
   floating-point operation count (FMA = 2) so that flops / elapsed time is the
   pipe throughput.  `sink` needs `blocks` elements of the chosen type. */
int bemppcuda_fma_probe(int32_t precision, int64_t iterations, int64_t blocks, void *sink, double *flops,
                        void *stream);

/* Shape derivatives of a DP0 Helmholtz scattering functional.  No single
   reference counterpart: the reference has no derivatives.  The operator is
       A = dlp_coeff * DLP + eta * SLP + identity * I        (DP0 x DP0, one grid)
   assembled by bemppcuda_assemble_regular (kernel BEMPPCUDA_HELMHOLTZ_COMBINED,
   params (k, 0, eta)) and bemppcuda_assemble_singular (diag_shift = identity);
   the far-field matrix is
       F[j, e] = ff_dlp_coeff * DLP_ff(d_j) + ff_eta * SLP_ff(d_j)
   with the kernels of helmholtz_far_field_{double,single}_layer
   (bempp_cl/core/numba_kernels.py:402-449); the right-hand side is
       b[e] = rhs_coeff * int_e exp(i k d_inc . x) dx
   with the regular rule (GridFunction projection onto DP0).  The wavenumber is
   real.  Quadrature points are fixed in reference coordinates, so the
   derivatives are exact derivatives of the discrete quantities. */
typedef struct {
    bemppcuda_grid grid;               /* geometry record of the (deformed) grid + elements */
    const int32_t *normal_mult;        /* (nelements,) DP0 normal multipliers; NULL means all +1 */
    double k;                          /* real wavenumber */
    double dlp_coeff;                  /* operator coefficients */
    double eta[2];
    double deta_dk[2];                 /* d eta / d k, e.g. -i for eta = -i k */
    double identity;
    int32_t nq;                        /* regular rule (6 points, order 4) */
    int32_t ndirections;               /* far-field directions */
    const double *quad_points;         /* HOST (nq, 2) */
    const double *quad_weights;        /* HOST (nq,) */
    /* Sauter-Schwab pairs of the DP0 space: every pair of elements sharing a vertex */
    int64_t npairs;
    const double *test_points;         /* (P, 2) */
    const double *trial_points;        /* (P, 2) */
    const double *weights;             /* (W,) */
    const int32_t *test_elements;      /* (npairs,) */
    const int32_t *trial_elements;
    const int32_t *test_offsets;
    const int32_t *trial_offsets;
    const int32_t *weights_offsets;
    const int32_t *npoints;
    /* far field */
    const double *directions;          /* (ndirections, 3) unit vectors */
    double ff_dlp_coeff;
    double ff_eta[2];
    double ff_deta_dk[2];
    /* right-hand side */
    double incident[3];                /* d_inc */
    double rhs_coeff[2];
    /* complex128 vectors */
    const void *phi;                   /* (nelements,) solution of A phi = b */
    const void *lambda;                /* (nelements,) adjoint solution of A^H lambda = F^H u */
    const void *u;                     /* (ndirections,) far field u = F phi */
    /* gradient contributions, each added with its scale:
         scale_operator * Re(lambda^H dA phi) + scale_farfield * Re(u^H dF phi)
       + scale_rhs * Re(lambda^H db) */
    double scale_operator;
    double scale_farfield;
    double scale_rhs;
    double *vertex_grad;               /* (nvertices, 3) accumulated (+=) */
    double *k_grad;                    /* (1,) accumulated (+=) */
    void *out;                         /* forward outputs: F (ndirections, nelements) row-major or b (nelements,) */
    void *workspace;                   /* >= bemppcuda_shape_workspace_bytes(nelements) */
    int64_t workspace_bytes;
    double phase_radius;               /* 2 x largest centroid-to-vertex distance, or 0 (unknown): when
                                          |k| * phase_radius <= 1 the phase offset k (r - r_c) of the
                                          regular pairs needs no range reduction */
} bemppcuda_shape_args;

int64_t bemppcuda_shape_workspace_bytes(int64_t nelements);

/* F[j, e] into args->out (complex128, ndirections x nelements). */
int bemppcuda_farfield_matrix_dp0(const bemppcuda_shape_args *args, void *stream);

/* b[e] into args->out (complex128, nelements). */
int bemppcuda_plane_wave_dp0(const bemppcuda_shape_args *args, void *stream);

/* Adds the vertex and wavenumber gradients of the three contractions above.
   The operator part never forms dA/dx: one pass over every regular element
   pair (quadrature recomputed, per-element partial sums in the workspace)
   and one over the singular pairs, then one per-element pass that applies
   the geometry chain rule and adds the far-field and right-hand-side terms. */
int bemppcuda_shape_adjoint_dp0(const bemppcuda_shape_args *args, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* BEMPPCUDA_H */
