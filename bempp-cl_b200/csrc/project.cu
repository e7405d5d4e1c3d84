// Projections of a function onto a scalar space: the device counterpart of
// GridFunction's vectorized projection (bempp_cl/api/assembly/grid_function.py,
// _project_function_vectorized): for every support element e and local shape
// function i,
//   P[l2g(e, i)] += mult(e, i) |J_e| sum_q w_q phi_i(q) f(e, q),
// f given at the regular rule's points of each support element.  Two steps,
// so that the function itself can be evaluated wherever it lives:
// bemppcuda_quadrature_points writes the global points and (normal-
// multiplied) unit normals of every (element, point) in the caller's
// vectorized layout (3, nsupport * nq), and bemppcuda_project forms the sums.
// One thread per (support element, shape function); the scatter into the
// zeroed output uses FP64 atomics (a dof is shared by the elements around it;
// the summation order is not fixed).
#include "common.cuh"

namespace bc {

__global__ void quadrature_points_kernel(const double *__restrict__ geom, int64_t ne,
                                         const uint32_t *__restrict__ support, int64_t nsup,
                                         const int32_t *__restrict__ nmult, QuadRule rule, double *points,
                                         double *normals) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = nsup * rule.nq;
    if (idx >= n) return;
    const int64_t k = idx / rule.nq;
    const int q = (int)(idx - k * rule.nq);
    const int64_t e = support[k];
    if (e >= ne) return;  // caller tables are not trusted
    Geom g;
    load_geom(geom, ne, e, nmult ? (double)nmult[e] : 1.0, g);
    double x[3];
    to_global(g, rule.x[q], rule.y[q], x);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        points[d * n + idx] = x[d];
        if (normals) normals[d * n + idx] = g.n[d];
    }
}

__global__ void project_kernel(const double *__restrict__ geom, int64_t ne, const uint32_t *__restrict__ support,
                               int64_t nsup, const uint32_t *__restrict__ l2g, const double *__restrict__ mult,
                               int nshape, int64_t ndofs, QuadRule rule, const double2 *__restrict__ values,
                               double2 *out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nsup * nshape) return;
    const int64_t k = idx / nshape;
    const int i = (int)(idx - k * nshape);
    const int64_t e = support[k];
    if (e >= ne) return;
    const double m = mult[e * nshape + i];
    const int64_t dof = l2g[e * nshape + i];
    if (m == 0.0 || dof >= ndofs) return;
    double sr = 0.0, si = 0.0;
    for (int q = 0; q < rule.nq; ++q) {
        const double w = nshape == 1 ? rule.w[q] : rule.sw[q][i];  // w_q phi_i(q)
        const double2 f = values[k * rule.nq + q];
        sr = fma(w, f.x, sr);
        si = fma(w, f.y, si);
    }
    const double s = m * __ldg(geom + 12 * ne + e);  // integration element
    double *o = reinterpret_cast<double *>(out + dof);
    atomicAdd(o, sr * s);
    atomicAdd(o + 1, si * s);
}

}  // namespace bc

using namespace bc;

static bool bad_projection_space(const bemppcuda_grid &g, const bemppcuda_space &s, int nq, const double *qp,
                                 const double *qw) {
    if (!g.geom || g.nelements < 0 || s.nsupport < 0 || (s.nsupport > 0 && !s.support)) {
        bc_set_error("projection: grid geometry or support missing");
        return true;
    }
    if (nq < 1 || nq > BEMPPCUDA_MAX_REGULAR_POINTS || !qp || !qw) {
        bc_set_error("projection: 1 <= nq <= %d host points and weights required", BEMPPCUDA_MAX_REGULAR_POINTS);
        return true;
    }
    return false;
}

extern "C" int bemppcuda_quadrature_points(const bemppcuda_grid *grid, const bemppcuda_space *space, int32_t nq,
                                           const double *quad_points, const double *quad_weights, double *points,
                                           double *normals, void *stream) {
    if (!grid || !space || bad_projection_space(*grid, *space, nq, quad_points, quad_weights)) {
        if (!grid || !space) bc_set_error("projection: null grid or space");
        return BEMPPCUDA_ERR_INVALID;
    }
    const int64_t n = space->nsupport * nq;
    if (n == 0) return BEMPPCUDA_OK;
    if (!points) {
        bc_set_error("quadrature_points: points missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    QuadRule rule;
    fill_rule(rule, nq, quad_points, quad_weights);
    quadrature_points_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        grid->geom, grid->nelements, space->support, space->nsupport, space->normal_mult, rule, points, normals);
    return bc_check_launch("quadrature_points");
}

extern "C" int bemppcuda_project(const bemppcuda_grid *grid, const bemppcuda_space *space, int32_t nq,
                                 const double *quad_points, const double *quad_weights, const void *values, void *out,
                                 void *stream) {
    if (!grid || !space || bad_projection_space(*grid, *space, nq, quad_points, quad_weights)) {
        if (!grid || !space) bc_set_error("projection: null grid or space");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (space->shapeset != BEMPPCUDA_SHAPE_P0 && space->shapeset != BEMPPCUDA_SHAPE_P1) {
        bc_set_error("project: scalar spaces (P0 / P1 shapesets) only");
        return BEMPPCUDA_ERR_UNSUPPORTED;
    }
    if ((space->shapeset == BEMPPCUDA_SHAPE_P0) != (space->nshape == 1) || !space->l2g || !space->mult ||
        space->ndofs < 0 || (space->ndofs > 0 && !out) || (space->nsupport > 0 && !values)) {
        bc_set_error("project: inconsistent space or missing values / output");
        return BEMPPCUDA_ERR_INVALID;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    if (space->ndofs > 0) {
        cudaError_t err = cudaMemsetAsync(out, 0, (size_t)space->ndofs * 16, st);
        if (err != cudaSuccess) {
            bc_set_error("project: %s", cudaGetErrorString(err));
            return BEMPPCUDA_ERR_CUDA;
        }
    }
    const int64_t n = space->nsupport * space->nshape;
    if (n == 0) return BEMPPCUDA_OK;
    QuadRule rule;
    fill_rule(rule, nq, quad_points, quad_weights);
    project_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(grid->geom, grid->nelements, space->support,
                                                                 space->nsupport, space->l2g, space->mult,
                                                                 space->nshape, space->ndofs, rule,
                                                                 static_cast<const double2 *>(values),
                                                                 static_cast<double2 *>(out));
    return bc_check_launch("project");
}
