// Potential and far-field evaluation: u(x) = sum over support elements and
// quadrature points of G(x, y_eq) c_eq.
//
// Replaces default_scalar_potential_kernel (numba_kernels.py:1788-1849),
// maxwell_efield_potential (:2281-2359), maxwell_mfield_potential
// (:2363-2433), maxwell_efield_far_field (:2437-2503) and
// maxwell_mfield_far_field (:2507-2570).
//
// Two launches on one stream:
//  1. potential_sources: one thread per (element, quadrature point) writes the
//     source point, normal and weighted coefficient(s) field-major into the
//     caller's workspace (the reference's `tmp` arrays).
//  2. potential_eval: one warp owns PPW evaluation points; its lanes stride
//     over the sources with coalesced loads, accumulate per point in FP64 and
//     combine with xor-shuffle reductions; lane 0 writes.
#include "common.cuh"

namespace bc {

// workspace fields per source
constexpr int SRC_FIELDS = 14;  // y(3) n(3) c0re c0im c1re c1im c2re c2im dre dim
constexpr int POT_PPW = 4;
constexpr int POT_WARPS = 4;

struct PotParams {
    const double *g;
    int64_t ne;
    const uint32_t *support;
    int64_t nsupport;
    const int32_t *nm;
    int nshape;
    int nq;
    const double *coeff;  // complex (ne * nshape)
    double *src;          // workspace SRC_FIELDS * nsrc
    int64_t nsrc;
    const double *points;  // (npoints, 3)
    int64_t npoints;
    double *result;  // complex (kdim, npoints)
    double p[4];
};

template <bool MAXWELL>
__global__ void potential_sources(PotParams prm, QuadRule rule) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= prm.nsrc) return;
    const int64_t ei = k / prm.nq;
    const int q = (int)(k - ei * prm.nq);
    const int64_t e = prm.support[ei];
    Geom g;
    load_geom(prm.g, prm.ne, e, prm.nm ? (double)prm.nm[e] : 1.0, g);
    double y[3];
    to_global(g, rule.x[q], rule.y[q], y);
    double *o = prm.src;
    const int64_t n = prm.nsrc;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        o[d * n + k] = y[d];
        o[(3 + d) * n + k] = g.n[d];
    }
    const double2 *x = reinterpret_cast<const double2 *>(prm.coeff) + e * prm.nshape;
    if (!MAXWELL) {
        double phi[3];
        scalar_shape(prm.nshape, rule.x[q], rule.y[q], phi);
        double cr = 0.0, ci = 0.0;
        for (int i = 0; i < prm.nshape; ++i) {
            const double2 xi = x[i];
            const double f = g.ie * rule.w[q] * phi[i];
            cr = fma(f, xi.x, cr);
            ci = fma(f, xi.y, ci);
        }
        o[6 * n + k] = cr;
        o[7 * n + k] = ci;
    } else {
        double b[3][3];
        rwg_values(g, rule.x[q], rule.y[q], b);
        double vr[3] = {0, 0, 0}, vi[3] = {0, 0, 0}, dr = 0.0, di = 0.0;
        for (int i = 0; i < 3; ++i) {
            const double2 xi = x[i];
            const double el = edge_length(prm.g, prm.ne, e, i);
            const double fr = rule.w[q] * xi.x * el, fi = rule.w[q] * xi.y * el;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                vr[d] += fr * b[i][d] * g.ie;
                vi[d] += fi * b[i][d] * g.ie;
            }
            dr += 2.0 * fr;
            di += 2.0 * fi;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            o[(6 + 2 * d) * n + k] = vr[d];
            o[(7 + 2 * d) * n + k] = vi[d];
        }
        o[12 * n + k] = dr;
        o[13 * n + k] = di;
    }
}

template <int ASM, int K>
__global__ void __launch_bounds__(32 * POT_WARPS) potential_eval(PotParams prm) {
    constexpr bool FAR = (K == BEMPPCUDA_FARFIELD_SLP || K == BEMPPCUDA_FARFIELD_DLP);
    constexpr int KD = (ASM == BEMPPCUDA_ASM_SCALAR) ? 1 : 3;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t)blockIdx.x * POT_WARPS + (threadIdx.x >> 5);
    const int64_t p0 = warp * POT_PPW;
    if (p0 >= prm.npoints) return;
    double xp[POT_PPW][3];
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j) {
        const int64_t pj = min(p0 + j, prm.npoints - 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) xp[j][d] = prm.points[3 * pj + d];
    }
    double ar[POT_PPW][KD], ai[POT_PPW][KD];
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j)
#pragma unroll
        for (int d = 0; d < KD; ++d) ar[j][d] = ai[j][d] = 0.0;
    const double kr = prm.p[0], ki = prm.p[1];
    const double zero[3] = {0.0, 0.0, 0.0};
    const int64_t n = prm.nsrc;
    const double *o = prm.src;
    for (int64_t k = lane; k < n; k += 32) {
        const double y[3] = {o[k], o[n + k], o[2 * n + k]};
        const double ny[3] = {o[3 * n + k], o[4 * n + k], o[5 * n + k]};
        if (ASM == BEMPPCUDA_ASM_SCALAR) {
            const double cr = o[6 * n + k], ci = o[7 * n + k];
#pragma unroll
            for (int j = 0; j < POT_PPW; ++j) {
                const cplx kv = greens<K>(xp[j], y, zero, ny, prm.p);
                ar[j][0] += kv.re * cr - kv.im * ci;
                ai[j][0] += kv.re * ci + kv.im * cr;
            }
        } else {
            cplx v[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) v[d] = {o[(6 + 2 * d) * n + k], o[(7 + 2 * d) * n + k]};
            const cplx dv = {o[12 * n + k], o[13 * n + k]};
            const cplx ik = {-ki, kr};
#pragma unroll
            for (int j = 0; j < POT_PPW; ++j) {
                const cplx kv = greens<K>(xp[j], y, zero, ny, prm.p);
                if (FAR) {
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const cplx t = cmul(ik, v[d]);
                            const cplx u = {t.re - xp[j][d] * dv.re, t.im - xp[j][d] * dv.im};
                            const cplx r = cmul(kv, u);
                            ar[j][d] += r.re;
                            ai[j][d] += r.im;
                        }
                    } else {
                        const cplx kik = cmul(kv, ik);
                        cplx val[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d) val[d] = cmul(kik, v[d]);
                        const double *x = xp[j];
                        ar[j][0] += x[1] * val[2].re - x[2] * val[1].re;
                        ai[j][0] += x[1] * val[2].im - x[2] * val[1].im;
                        ar[j][1] += x[2] * val[0].re - x[0] * val[2].re;
                        ai[j][1] += x[2] * val[0].im - x[0] * val[2].im;
                        ar[j][2] += x[0] * val[1].re - x[1] * val[0].re;
                        ai[j][2] += x[0] * val[1].im - x[1] * val[0].im;
                    }
                } else {
                    const double df[3] = {xp[j][0] - y[0], xp[j][1] - y[1], xp[j][2] - y[2]};
                    const double dist2 = df[0] * df[0] + df[1] * df[1] + df[2] * df[2];
                    const double dist = sqrt(dist2);
                    const cplx ikd1 = {-ki * dist - 1.0, kr * dist};  // i k dist - 1
                    if (ASM == BEMPPCUDA_ASM_EFIE) {
                        // (i k d - 1) dv / (i k d^2)
                        const cplx ikd2 = {-ki * dist2, kr * dist2};
                        const double den = ikd2.re * ikd2.re + ikd2.im * ikd2.im;
                        const cplx num = cmul(ikd1, dv);
                        const cplx q = {(num.re * ikd2.re + num.im * ikd2.im) / den,
                                        (num.im * ikd2.re - num.re * ikd2.im) / den};
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const cplx t = cmul(ik, v[d]);
                            const cplx u = {t.re - df[d] * q.re, t.im - df[d] * q.im};
                            const cplx r = cmul(kv, u);
                            ar[j][d] += r.re;
                            ai[j][d] += r.im;
                        }
                    } else {
                        const cplx f = cscale(cmul(kv, ikd1), 1.0 / dist2);
                        cplx val[3];
#pragma unroll
                        for (int d = 0; d < 3; ++d) val[d] = cmul(f, v[d]);
                        ar[j][0] += df[1] * val[2].re - df[2] * val[1].re;
                        ai[j][0] += df[1] * val[2].im - df[2] * val[1].im;
                        ar[j][1] += df[2] * val[0].re - df[0] * val[2].re;
                        ai[j][1] += df[2] * val[0].im - df[0] * val[2].im;
                        ar[j][2] += df[0] * val[1].re - df[1] * val[0].re;
                        ai[j][2] += df[0] * val[1].im - df[1] * val[0].im;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < POT_PPW; ++j)
#pragma unroll
        for (int d = 0; d < KD; ++d) {
            ar[j][d] = warp_sum(ar[j][d]);
            ai[j][d] = warp_sum(ai[j][d]);
        }
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < POT_PPW; ++j) {
            const int64_t pj = p0 + j;
            if (pj >= prm.npoints) break;
#pragma unroll
            for (int d = 0; d < KD; ++d) {
                prm.result[2 * (d * prm.npoints + pj)] = ar[j][d];
                prm.result[2 * (d * prm.npoints + pj) + 1] = ai[j][d];
            }
        }
    }
}

template <int ASM, int K>
static cudaError_t launch_pot(const PotParams &prm, cudaStream_t st) {
    const int64_t warps = (prm.npoints + POT_PPW - 1) / POT_PPW;
    const unsigned blocks = (unsigned)((warps + POT_WARPS - 1) / POT_WARPS);
    potential_eval<ASM, K><<<blocks, 32 * POT_WARPS, 0, st>>>(prm);
    return cudaGetLastError();
}

}  // namespace bc

using namespace bc;

int64_t bc_potential_workspace_doubles(int64_t nsupport, int nq) { return (int64_t)SRC_FIELDS * nsupport * nq; }

// `workspace` must hold bc_potential_workspace_doubles() doubles.
int bc_potential_launch(const bemppcuda_potential_args *a, double *workspace, cudaStream_t st) {
    PotParams prm;
    prm.g = a->grid.geom;
    prm.ne = a->grid.nelements;
    prm.support = a->space.support;
    prm.nsupport = a->space.nsupport;
    prm.nm = a->space.normal_mult;
    prm.nshape = a->space.nshape;
    prm.nq = a->nq;
    prm.coeff = a->coefficients;
    prm.src = workspace;
    prm.nsrc = a->space.nsupport * a->nq;
    prm.points = a->points;
    prm.npoints = a->npoints;
    prm.result = reinterpret_cast<double *>(a->result);
    for (int i = 0; i < 4; ++i) prm.p[i] = a->params[i];
    QuadRule rule;
    rule.nq = a->nq;
    rule.pad = 0;
    for (int i = 0; i < BEMPPCUDA_MAX_REGULAR_POINTS; ++i) {
        rule.x[i] = i < a->nq ? a->quad_points[2 * i] : 0.0;
        rule.y[i] = i < a->nq ? a->quad_points[2 * i + 1] : 0.0;
        rule.w[i] = i < a->nq ? a->quad_weights[i] : 0.0;
        rule.wf[i] = (float)rule.w[i];
    }
    if (prm.npoints == 0) return BEMPPCUDA_OK;
    const bool maxwell = a->assembly != BEMPPCUDA_ASM_SCALAR;
    if (prm.nsrc > 0) {
        const unsigned blocks = (unsigned)((prm.nsrc + 255) / 256);
        if (maxwell)
            potential_sources<true><<<blocks, 256, 0, st>>>(prm, rule);
        else
            potential_sources<false><<<blocks, 256, 0, st>>>(prm, rule);
    }
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) {
        if (!maxwell) {
            switch (a->kernel) {
            case BEMPPCUDA_LAPLACE_SLP: err = launch_pot<0, BEMPPCUDA_LAPLACE_SLP>(prm, st); break;
            case BEMPPCUDA_LAPLACE_DLP: err = launch_pot<0, BEMPPCUDA_LAPLACE_DLP>(prm, st); break;
            case BEMPPCUDA_HELMHOLTZ_SLP: err = launch_pot<0, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st); break;
            case BEMPPCUDA_HELMHOLTZ_DLP: err = launch_pot<0, BEMPPCUDA_HELMHOLTZ_DLP>(prm, st); break;
            case BEMPPCUDA_MODHELM_SLP: err = launch_pot<0, BEMPPCUDA_MODHELM_SLP>(prm, st); break;
            case BEMPPCUDA_MODHELM_DLP: err = launch_pot<0, BEMPPCUDA_MODHELM_DLP>(prm, st); break;
            case BEMPPCUDA_FARFIELD_SLP: err = launch_pot<0, BEMPPCUDA_FARFIELD_SLP>(prm, st); break;
            case BEMPPCUDA_FARFIELD_DLP: err = launch_pot<0, BEMPPCUDA_FARFIELD_DLP>(prm, st); break;
            default: bc_set_error("kernel %d not valid for a scalar potential", a->kernel); return BEMPPCUDA_ERR_INVALID;
            }
        } else {
            const bool far = a->kernel == BEMPPCUDA_FARFIELD_SLP;
            if (a->kernel != BEMPPCUDA_HELMHOLTZ_SLP && !far) {
                bc_set_error("Maxwell potentials use the Helmholtz single-layer kernel (got %d)", a->kernel);
                return BEMPPCUDA_ERR_INVALID;
            }
            if (a->assembly == BEMPPCUDA_ASM_EFIE)
                err = far ? launch_pot<4, BEMPPCUDA_FARFIELD_SLP>(prm, st) : launch_pot<4, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st);
            else if (a->assembly == BEMPPCUDA_ASM_MFIE)
                err = far ? launch_pot<5, BEMPPCUDA_FARFIELD_SLP>(prm, st) : launch_pot<5, BEMPPCUDA_HELMHOLTZ_SLP>(prm, st);
            else {
                bc_set_error("assembly type %d not valid for a potential", a->assembly);
                return BEMPPCUDA_ERR_INVALID;
            }
        }
    }
    if (err != cudaSuccess) {
        bc_set_error("potential launch failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    return BEMPPCUDA_OK;
}
