// C-ABI entry points: argument validation, per-thread error messages and the
// element geometry kernel.  Declarations and field documentation live in
// include/bemppcuda.h.
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "common.cuh"

int bc_regular_launch(const bemppcuda_regular_args *a, cudaStream_t st);
int bc_apply_launch(const bemppcuda_regular_args *a, const void *x, void *y, cudaStream_t st);
int bc_singular_launch(const bemppcuda_singular_args *a, cudaStream_t st);
int bc_potential_launch(const bemppcuda_potential_args *a, double *workspace, cudaStream_t st);
int64_t bc_potential_workspace_doubles(int64_t nsupport, int nq);

static thread_local char g_error[1024] = "";

void bc_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

int bc_check_launch(const char *what) {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        bc_set_error("%s: %s", what, cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}

namespace bc {

// Per-element geometry (grid.py:552-590): Jacobian columns, unit normal,
// integration element sqrt(det(J^T J)), edge lengths, J (J^T J)^-1, centroid.
__global__ void grid_geometry_kernel(const double *__restrict__ v, int64_t nv, const int32_t *__restrict__ el,
                                     int64_t ne, double *__restrict__ g, int *__restrict__ bad) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int i0 = el[3 * e], i1 = el[3 * e + 1], i2 = el[3 * e + 2];
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= nv || i1 >= nv || i2 >= nv) {
        atomicExch(bad, 1);
        for (int f = 0; f < BEMPPCUDA_GEOM_FIELDS; ++f) g[f * ne + e] = 0.0;
        return;
    }
    double a[3], b[3], c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        a[d] = v[3 * (int64_t)i0 + d];
        b[d] = v[3 * (int64_t)i1 + d];
        c[d] = v[3 * (int64_t)i2 + d];
    }
    double j0[3], j1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        j0[d] = b[d] - a[d];
        j1[d] = c[d] - a[d];
    }
    const double cr[3] = {j0[1] * j1[2] - j0[2] * j1[1], j0[2] * j1[0] - j0[0] * j1[2], j0[0] * j1[1] - j0[1] * j1[0]};
    const double nn = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    const double m00 = j0[0] * j0[0] + j0[1] * j0[1] + j0[2] * j0[2];
    const double m01 = j0[0] * j1[0] + j0[1] * j1[1] + j0[2] * j1[2];
    const double m11 = j1[0] * j1[0] + j1[1] * j1[1] + j1[2] * j1[2];
    const double det = m00 * m11 - m01 * m01;
    if (!(nn > 0.0) || !(det > 0.0)) atomicExch(bad, 2);
    const double i00 = m11 / det, i11 = m00 / det, i01 = -m01 / det;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g[(0 + d) * ne + e] = a[d];
        g[(3 + d) * ne + e] = j0[d];
        g[(6 + d) * ne + e] = j1[d];
        g[(9 + d) * ne + e] = cr[d] / nn;
        g[(16 + 2 * d) * ne + e] = j0[d] * i00 + j1[d] * i01;
        g[(17 + 2 * d) * ne + e] = j0[d] * i01 + j1[d] * i11;
        g[(22 + d) * ne + e] = (a[d] + b[d] + c[d]) / 3.0;
    }
    g[12 * ne + e] = sqrt(det);
    double e0 = 0, e1 = 0, e2 = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        e0 += (a[d] - b[d]) * (a[d] - b[d]);
        e1 += (c[d] - a[d]) * (c[d] - a[d]);
        e2 += (b[d] - c[d]) * (b[d] - c[d]);
    }
    g[13 * ne + e] = sqrt(e0);
    g[14 * ne + e] = sqrt(e1);
    g[15 * ne + e] = sqrt(e2);
}

}  // namespace bc

static bool bad_space(const bemppcuda_space &s, const char *name, bool need_maps) {
    if (s.nshape != 1 && s.nshape != 3) {
        bc_set_error("%s: nshape must be 1 or 3 (got %d)", name, s.nshape);
        return true;
    }
    if (s.nsupport < 0 || (s.nsupport > 0 && !s.support)) {
        bc_set_error("%s: support pointer missing", name);
        return true;
    }
    if (need_maps && (!s.l2g || !s.mult)) {
        bc_set_error("%s: local2global / multipliers missing", name);
        return true;
    }
    if (s.shapeset == BEMPPCUDA_SHAPE_P0 && s.nshape != 1) {
        bc_set_error("%s: p0 shapeset needs nshape 1", name);
        return true;
    }
    return false;
}

static bool bad_grid(const bemppcuda_grid &g, const char *name) {
    if (g.nelements < 0 || (g.nelements > 0 && (!g.geom || !g.elements))) {
        bc_set_error("%s: geometry / elements missing", name);
        return true;
    }
    return false;
}

static bool bad_params(const double *p, int kernel, int assembly) {
    for (int i = 0; i < 4; ++i)
        if (!(p[i] == p[i]) || p[i] > 1e300 || p[i] < -1e300) {
            bc_set_error("kernel parameters must be finite");
            return true;
        }
    const bool helm = (kernel == BEMPPCUDA_HELMHOLTZ_SLP || kernel == BEMPPCUDA_HELMHOLTZ_DLP ||
                       kernel == BEMPPCUDA_HELMHOLTZ_ADLP || assembly == BEMPPCUDA_ASM_EFIE ||
                       assembly == BEMPPCUDA_ASM_MFIE);
    if (helm && p[0] == 0.0 && p[1] == 0.0 && (assembly == BEMPPCUDA_ASM_EFIE || assembly == BEMPPCUDA_ASM_MFIE)) {
        bc_set_error("Maxwell operators need a nonzero wavenumber");
        return true;
    }
    return false;
}

extern "C" {

int bemppcuda_version(void) { return 100; }

int bemppcuda_last_error(char *buffer, int64_t length) {
    if (!buffer || length <= 0) return BEMPPCUDA_ERR_INVALID;
    snprintf(buffer, (size_t)length, "%s", g_error);
    return BEMPPCUDA_OK;
}

int bemppcuda_grid_geometry(const double *vertices, int64_t nvertices, const int32_t *elements, int64_t nelements,
                            double *geom, void *stream) {
    if (nelements < 0 || nvertices < 0) {
        bc_set_error("negative grid size");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (nelements == 0) return BEMPPCUDA_OK;
    if (!vertices || !elements || !geom) {
        bc_set_error("grid_geometry: null pointer");
        return BEMPPCUDA_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // one 4-byte check word per device, allocated on first use and kept
    static int *d_flags[256] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        bc_set_error("grid_geometry: no usable CUDA device");
        return BEMPPCUDA_ERR_CUDA;
    }
    if (!d_flags[dev] && cudaMalloc(&d_flags[dev], sizeof(int)) != cudaSuccess) {
        d_flags[dev] = nullptr;
        bc_set_error("grid_geometry: cannot allocate the check word");
        return BEMPPCUDA_ERR_CUDA;
    }
    int *d_flag = d_flags[dev];
    cudaMemsetAsync(d_flag, 0, sizeof(int), st);
    const unsigned blocks = (unsigned)((nelements + 127) / 128);
    bc::grid_geometry_kernel<<<blocks, 128, 0, st>>>(vertices, nvertices, elements, nelements, geom, d_flag);
    int rc = bc_check_launch("grid_geometry");
    if (rc) return rc;
    int h_flag = 0;
    if (cudaMemcpyAsync(&h_flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        bc_set_error("grid_geometry: %s", cudaGetErrorString(cudaGetLastError()));
        return BEMPPCUDA_ERR_CUDA;
    }
    if (h_flag == 1) {
        bc_set_error("grid_geometry: element vertex index out of range");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (h_flag == 2) {
        bc_set_error("grid_geometry: degenerate element (zero area) or non-finite vertex");
        return BEMPPCUDA_ERR_INVALID;
    }
    return BEMPPCUDA_OK;
}

int bemppcuda_assemble_regular(const bemppcuda_regular_args *a, void *stream) {
    if (!a) {
        bc_set_error("null argument struct");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (bad_grid(a->test_grid, "test grid") || bad_grid(a->trial_grid, "trial grid")) return BEMPPCUDA_ERR_INVALID;
    if (bad_space(a->test, "test space", true) || bad_space(a->trial, "trial space", true)) return BEMPPCUDA_ERR_INVALID;
    if (bad_params(a->params, a->kernel, a->assembly)) return BEMPPCUDA_ERR_INVALID;
    if (a->nq < 1 || a->nq > BEMPPCUDA_MAX_REGULAR_POINTS || !a->quad_points || !a->quad_weights) {
        bc_set_error("regular rule: 1 <= nq <= %d host points and weights required", BEMPPCUDA_MAX_REGULAR_POINTS);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (!a->result || a->ld < a->trial.ndofs - (a->tresult ? a->col_begin : 0)) {
        bc_set_error("result pointer missing or ld (%lld) < columns (%lld)", (long long)a->ld,
                     (long long)a->trial.ndofs);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->precision != BEMPPCUDA_FP64 && a->precision != BEMPPCUDA_MIXED) {
        bc_set_error("precision must be BEMPPCUDA_FP64 or BEMPPCUDA_MIXED");
        return BEMPPCUDA_ERR_INVALID;
    }
    if ((a->assembly == BEMPPCUDA_ASM_EFIE || a->assembly == BEMPPCUDA_ASM_MFIE) &&
        (a->test.shapeset != BEMPPCUDA_SHAPE_RWG || a->trial.shapeset != BEMPPCUDA_SHAPE_RWG)) {
        bc_set_error("Maxwell assembly needs RWG/SNC spaces on both sides");
        return BEMPPCUDA_ERR_INVALID;
    }
    if ((a->assembly >= BEMPPCUDA_ASM_LAPLACE_HYP && a->assembly <= BEMPPCUDA_ASM_MODHELM_HYP) &&
        (a->test.nshape != 3 || a->trial.nshape != 3)) {
        bc_set_error("hypersingular assembly needs p1_discontinuous shapesets on both sides");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (!a->is_complex && ((a->kernel >= BEMPPCUDA_HELMHOLTZ_SLP && a->kernel <= BEMPPCUDA_HELMHOLTZ_ADLP) ||
                           a->kernel == BEMPPCUDA_HELMHOLTZ_COMBINED)) {
        bc_set_error("Helmholtz kernels need a complex result");
        return BEMPPCUDA_ERR_INVALID;
    }
    return bc_regular_launch(a, (cudaStream_t)stream);
}

int bemppcuda_apply_regular(const bemppcuda_regular_args *a, const void *x, void *y, void *stream) {
    if (!a) {
        bc_set_error("null argument struct");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (bad_grid(a->test_grid, "test grid") || bad_grid(a->trial_grid, "trial grid")) return BEMPPCUDA_ERR_INVALID;
    if (bad_space(a->test, "test space", true) || bad_space(a->trial, "trial space", true)) return BEMPPCUDA_ERR_INVALID;
    if (bad_params(a->params, a->kernel, a->assembly)) return BEMPPCUDA_ERR_INVALID;
    if (a->nq < 1 || a->nq > BEMPPCUDA_MAX_REGULAR_POINTS || !a->quad_points || !a->quad_weights) {
        bc_set_error("regular rule: 1 <= nq <= %d host points and weights required", BEMPPCUDA_MAX_REGULAR_POINTS);
        return BEMPPCUDA_ERR_INVALID;
    }
    if ((a->trial.nsupport > 0 && !x) || (a->test.nsupport > 0 && !y)) {
        bc_set_error("apply_regular: x / y missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    return bc_apply_launch(a, x, y, (cudaStream_t)stream);
}

int bemppcuda_assemble_singular(const bemppcuda_singular_args *a, void *stream) {
    if (!a) {
        bc_set_error("null argument struct");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (bad_grid(a->grid, "grid")) return BEMPPCUDA_ERR_INVALID;
    if (bad_space(a->test, "test space", a->dense != nullptr) || bad_space(a->trial, "trial space", a->dense != nullptr))
        return BEMPPCUDA_ERR_INVALID;
    if (bad_params(a->params, a->kernel, a->assembly)) return BEMPPCUDA_ERR_INVALID;
    if ((a->values == nullptr) == (a->dense == nullptr)) {
        bc_set_error("exactly one of values / dense must be given");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->npairs < 0 || (a->npairs > 0 && (!a->test_points || !a->trial_points || !a->weights ||
                                            !a->test_elements || !a->trial_elements || !a->test_offsets ||
                                            !a->trial_offsets || !a->weights_offsets || !a->npoints))) {
        bc_set_error("singular pair arrays missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->dense && a->ld < a->trial.ndofs) {
        bc_set_error("dense ld smaller than the column count");
        return BEMPPCUDA_ERR_INVALID;
    }
    return bc_singular_launch(a, (cudaStream_t)stream);
}

int64_t bemppcuda_potential_workspace_bytes(const bemppcuda_potential_args *a) {
    if (!a || a->space.nsupport < 0 || a->nq < 1) return 0;
    const int64_t doubles = bc_potential_workspace_doubles(a->space.nsupport, a->nq);
    return (doubles < 0 || doubles > INT64_MAX / 8) ? -1 : 8 * doubles;
}

int bemppcuda_evaluate_potential(const bemppcuda_potential_args *a, void *stream) {
    if (!a) {
        bc_set_error("null argument struct");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (bad_grid(a->grid, "grid") || bad_space(a->space, "space", false)) return BEMPPCUDA_ERR_INVALID;
    if (bad_params(a->params, a->kernel, a->assembly)) return BEMPPCUDA_ERR_INVALID;
    if (a->nq < 1 || a->nq > BEMPPCUDA_MAX_REGULAR_POINTS || !a->quad_points || !a->quad_weights) {
        bc_set_error("potential rule: 1 <= nq <= %d host points and weights required", BEMPPCUDA_MAX_REGULAR_POINTS);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->npoints < 0 || (a->npoints > 0 && (!a->points || !a->result))) {
        bc_set_error("points / result missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->space.nsupport > 0 && !a->coefficients) {
        bc_set_error("coefficients missing");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->assembly != BEMPPCUDA_ASM_SCALAR && a->space.shapeset != BEMPPCUDA_SHAPE_RWG) {
        bc_set_error("Maxwell potentials need an RWG space");
        return BEMPPCUDA_ERR_INVALID;
    }
    const int64_t need = bemppcuda_potential_workspace_bytes(a);
    if (need < 0) {
        bc_set_error("potential: %lld support elements x %d points overflow the workspace size",
                     (long long)a->space.nsupport, a->nq);
        return BEMPPCUDA_ERR_INVALID;
    }
    if (need > 0 && (!a->workspace || a->workspace_bytes < need)) {
        bc_set_error("potential workspace too small: need %lld bytes, got %lld", (long long)need,
                     (long long)a->workspace_bytes);
        return BEMPPCUDA_ERR_WORKSPACE;
    }
    return bc_potential_launch(a, reinterpret_cast<double *>(a->workspace), (cudaStream_t)stream);
}

}  // extern "C"
