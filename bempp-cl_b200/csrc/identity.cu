// L2 identity (mass matrix) of two spaces on one grid, as COO triplets: the
// device counterpart of l2_identity_kernel (numba_kernels.py:713-769) driven by
// default_sparse_kernel (:935-976) and SparseAssembler.assemble
// (core/sparse_assembler.py:17-70).
//
// For every element e in both supports and local functions i (test), j
// (trial):
//   value = m_t(e, i) m_s(e, j) |J_e| sum_q w_q phi_i(q) . psi_j(q)
//   row = l2g_t(e, i), col = l2g_s(e, j)
// The reference evaluates the basis of the localised spaces (multipliers 1 on
// the support) and multiplies by the spaces' own multipliers afterwards; the
// product is the same.  Basis values: P0 1; P1 / DP1 (1 - xi - eta, xi, eta);
// RWG l_i / |J| J r_i(xi, eta) (maxwell_spaces.py:678-712, l_i the edge
// length, r_i the reference functions of shapesets.py:95-102); SNC the RWG
// value turned by the element normal, n x b_i (maxwell_spaces.py:716-757, n
// times the normal multiplier).  Duplicated (row, col) pairs are summed by the
// caller when it builds the sparse matrix, as scipy's coo_matrix.tocsr() does
// in the reference.  One thread per element; the work is O(elements).
#include "common.cuh"

namespace bc {

struct IdParams {
    const double *g;
    int64_t ne;
    const uint32_t *elements;
    int64_t nel;
    const uint32_t *tl2g, *sl2g;
    const double *tmult, *smult;
    const int32_t *tnm, *snm;
    int64_t *rows, *cols;
    double *values;
};

// values of the NB functions of kind KIND at reference point (x, y), dimension D (1 scalar, 3 vector)
template <int KIND, int NB>
__device__ __forceinline__ void id_basis(const Geom &g, const double el[3], double nmul, double x, double y,
                                         double v[3][3]) {
    if (KIND == BEMPPCUDA_BASIS_SCALAR) {
        double s[3];
        scalar_shape(NB, x, y, s);
#pragma unroll
        for (int i = 0; i < 3; ++i) v[i][0] = s[i];
    } else {
        double b[3][3];
        rwg_values(g, x, y, b);  // J r_i / |J|
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int d = 0; d < 3; ++d) b[i][d] *= el[i];
            if (KIND == BEMPPCUDA_BASIS_SNC) {
                const double n0 = g.n[0] * nmul, n1 = g.n[1] * nmul, n2 = g.n[2] * nmul;
                v[i][0] = n1 * b[i][2] - n2 * b[i][1];
                v[i][1] = n2 * b[i][0] - n0 * b[i][2];
                v[i][2] = n0 * b[i][1] - n1 * b[i][0];
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) v[i][d] = b[i][d];
            }
        }
    }
}

template <int KT, int NT, int KS, int NS>
__global__ void __launch_bounds__(128) identity_coo(IdParams prm, QuadRule rule, int nq) {
    constexpr int D = (KT == BEMPPCUDA_BASIS_SCALAR) ? 1 : 3;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= prm.nel) return;
    const int64_t e = prm.elements[idx];
    Geom g;
    load_geom(prm.g, prm.ne, e, 1.0, g);
    double el[3] = {1.0, 1.0, 1.0};
    if (KT != BEMPPCUDA_BASIS_SCALAR)
#pragma unroll
        for (int i = 0; i < 3; ++i) el[i] = edge_length(prm.g, prm.ne, e, i);
    const double tn = prm.tnm ? (double)prm.tnm[e] : 1.0, sn = prm.snm ? (double)prm.snm[e] : 1.0;
    double blk[NT][NS];
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) blk[i][j] = 0.0;
    for (int q = 0; q < nq; ++q) {
        double vt[3][3] = {}, vs[3][3] = {};
        id_basis<KT, NT>(g, el, tn, rule.x[q], rule.y[q], vt);
        id_basis<KS, NS>(g, el, sn, rule.x[q], rule.y[q], vs);
        const double w = rule.w[q];
#pragma unroll
        for (int i = 0; i < NT; ++i)
#pragma unroll
            for (int j = 0; j < NS; ++j) {
                double dot = 0.0;
#pragma unroll
                for (int d = 0; d < D; ++d) dot = fma(vt[i][d], vs[j][d], dot);
                blk[i][j] = fma(w, dot, blk[i][j]);
            }
    }
    const int64_t base = idx * NT * NS;
#pragma unroll
    for (int i = 0; i < NT; ++i)
#pragma unroll
        for (int j = 0; j < NS; ++j) {
            const int64_t o = base + i * NS + j;
            prm.rows[o] = prm.tl2g[e * NT + i];
            prm.cols[o] = prm.sl2g[e * NS + j];
            prm.values[o] = blk[i][j] * g.ie * prm.tmult[e * NT + i] * prm.smult[e * NS + j];
        }
}

template <int KT, int NT, int KS, int NS>
static cudaError_t launch_identity(const IdParams &prm, const QuadRule &rule, int nq, cudaStream_t st) {
    const unsigned blocks = (unsigned)((prm.nel + 127) / 128);
    identity_coo<KT, NT, KS, NS><<<blocks, 128, 0, st>>>(prm, rule, nq);
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

extern "C" int bemppcuda_assemble_identity(const bemppcuda_identity_args *a, void *stream) {
    if (!a || !a->grid.geom || a->nelements < 0 || (a->nelements > 0 && (!a->elements || !a->rows || !a->cols ||
                                                                          !a->values))) {
        bc_set_error("identity: missing grid, element list or outputs");
        return BEMPPCUDA_ERR_INVALID;
    }
    const int tk = a->test_kind, sk = a->trial_kind, nt = a->test.nshape, ns = a->trial.nshape;
    const bool t_vec = tk == BEMPPCUDA_BASIS_RWG || tk == BEMPPCUDA_BASIS_SNC;
    const bool s_vec = sk == BEMPPCUDA_BASIS_RWG || sk == BEMPPCUDA_BASIS_SNC;
    if ((tk != BEMPPCUDA_BASIS_SCALAR && !t_vec) || (sk != BEMPPCUDA_BASIS_SCALAR && !s_vec) || t_vec != s_vec ||
        (nt != 1 && nt != 3) || (ns != 1 && ns != 3) || (t_vec && (nt != 3 || ns != 3))) {
        bc_set_error("identity: test / trial bases must both be scalar (1 or 3 functions) or both RWG / SNC");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (!a->test.l2g || !a->trial.l2g || !a->test.mult || !a->trial.mult) {
        bc_set_error("identity: dof maps missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->nq < 1 || a->nq > BEMPPCUDA_MAX_REGULAR_POINTS || !a->quad_points || !a->quad_weights) {
        bc_set_error("identity: quadrature rule must have 1..%d points", BEMPPCUDA_MAX_REGULAR_POINTS);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->nelements == 0) return BEMPPCUDA_OK;
    IdParams prm;
    prm.g = a->grid.geom;
    prm.ne = a->grid.nelements;
    prm.elements = a->elements;
    prm.nel = a->nelements;
    prm.tl2g = a->test.l2g;
    prm.sl2g = a->trial.l2g;
    prm.tmult = a->test.mult;
    prm.smult = a->trial.mult;
    prm.tnm = a->test.normal_mult;
    prm.snm = a->trial.normal_mult;
    prm.rows = a->rows;
    prm.cols = a->cols;
    prm.values = a->values;
    QuadRule rule;
    fill_rule(rule, a->nq, a->quad_points, a->quad_weights);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err;
    constexpr int S = BEMPPCUDA_BASIS_SCALAR, R = BEMPPCUDA_BASIS_RWG, C = BEMPPCUDA_BASIS_SNC;
    if (!t_vec) {
        if (nt == 1 && ns == 1)
            err = launch_identity<S, 1, S, 1>(prm, rule, a->nq, st);
        else if (nt == 1)
            err = launch_identity<S, 1, S, 3>(prm, rule, a->nq, st);
        else if (ns == 1)
            err = launch_identity<S, 3, S, 1>(prm, rule, a->nq, st);
        else
            err = launch_identity<S, 3, S, 3>(prm, rule, a->nq, st);
    } else if (tk == R && sk == R) {
        err = launch_identity<R, 3, R, 3>(prm, rule, a->nq, st);
    } else if (tk == R) {
        err = launch_identity<R, 3, C, 3>(prm, rule, a->nq, st);
    } else if (sk == R) {
        err = launch_identity<C, 3, R, 3>(prm, rule, a->nq, st);
    } else {
        err = launch_identity<C, 3, C, 3>(prm, rule, a->nq, st);
    }
    if (err != cudaSuccess) {
        bc_set_error("identity launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
