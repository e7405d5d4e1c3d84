/*
 * CPU oracle for the dense Galerkin assembly and potential path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C (OpenMP) restatement of
 * the reference Numba kernels, used by the tests, the smoke check and the CPU
 * baseline leg of bench.py as the checker.  The product never links, loads or
 * calls it.
 *
 * Every routine follows one reference function, cited by file:line inside
 * bempp_cl/core/numba_kernels.py unless stated otherwise.  All arithmetic is
 * double precision, as the reference does regardless of the requested
 * precision (numba_assemblers.py:30-32, 72-74, 127-129).
 *
 * Geometry is recomputed here from vertices and elements (grid.py:552-590):
 * v0 = vertex 0, jacobian columns v1 - v0 and v2 - v0, unit normal
 * (cross product) times the space's normal multiplier, integration element
 * sqrt(det(J^T J)) and J (J^T J)^-1 for surface gradients.
 *
 * Result buffers use numpy's layout: row-major (rows, cols), complex numbers
 * as interleaved (re, im) doubles.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define M_INV_4PI_D (1.0 / (4.0 * 3.14159265358979323846))

enum {
    ORC_LAPLACE_SLP = 0,
    ORC_LAPLACE_DLP = 1,
    ORC_LAPLACE_ADLP = 2,
    ORC_HELMHOLTZ_SLP = 3,
    ORC_HELMHOLTZ_DLP = 4,
    ORC_HELMHOLTZ_ADLP = 5,
    ORC_MODHELM_SLP = 6,
    ORC_MODHELM_DLP = 7,
    ORC_MODHELM_ADLP = 8,
    ORC_FARFIELD_SLP = 9,
    ORC_FARFIELD_DLP = 10,
    ORC_HELMHOLTZ_COMBINED = 11
};

enum { ORC_ASM_SCALAR = 0, ORC_ASM_LAPLACE_HYP = 1, ORC_ASM_HELM_HYP = 2, ORC_ASM_MODHELM_HYP = 3,
       ORC_ASM_EFIE = 4, ORC_ASM_MFIE = 5 };

typedef struct {
    double v0[3];
    double j[3][2];
    double n[3];
    double ie;
    double jit[3][2];
    double el[3]; /* edge lengths |v0-v1|, |v2-v0|, |v1-v2| (numba_kernels.py:114-133) */
} elem_geom;

static void geom(const double *vertices, int64_t nv, const uint32_t *elements, int64_t ne, int64_t e,
                 double normal_mult, elem_geom *g) {
    /* vertices: (3, nv) Fortran order, i.e. vertices[d + 3 * v]
       elements: (3, ne) Fortran order, elements[k + 3 * e] */
    (void)nv;
    (void)ne;
    const double *a = vertices + 3 * (int64_t)elements[0 + 3 * e];
    const double *b = vertices + 3 * (int64_t)elements[1 + 3 * e];
    const double *c = vertices + 3 * (int64_t)elements[2 + 3 * e];
    for (int d = 0; d < 3; ++d) {
        g->v0[d] = a[d];
        g->j[d][0] = b[d] - a[d];
        g->j[d][1] = c[d] - a[d];
    }
    double cr[3] = {g->j[1][0] * g->j[2][1] - g->j[2][0] * g->j[1][1],
                    g->j[2][0] * g->j[0][1] - g->j[0][0] * g->j[2][1],
                    g->j[0][0] * g->j[1][1] - g->j[1][0] * g->j[0][1]};
    double nn = sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
    for (int d = 0; d < 3; ++d) g->n[d] = cr[d] / nn * normal_mult;
    double m00 = 0, m01 = 0, m11 = 0;
    for (int d = 0; d < 3; ++d) {
        m00 += g->j[d][0] * g->j[d][0];
        m01 += g->j[d][0] * g->j[d][1];
        m11 += g->j[d][1] * g->j[d][1];
    }
    double det = m00 * m11 - m01 * m01;
    g->ie = sqrt(det);
    double i00 = m11 / det, i11 = m00 / det, i01 = -m01 / det;
    for (int d = 0; d < 3; ++d) {
        g->jit[d][0] = g->j[d][0] * i00 + g->j[d][1] * i01;
        g->jit[d][1] = g->j[d][0] * i01 + g->j[d][1] * i11;
    }
    double e0 = 0, e1 = 0, e2 = 0;
    for (int d = 0; d < 3; ++d) {
        e0 += (a[d] - b[d]) * (a[d] - b[d]);
        e1 += (c[d] - a[d]) * (c[d] - a[d]);
        e2 += (b[d] - c[d]) * (b[d] - c[d]);
    }
    g->el[0] = sqrt(e0);
    g->el[1] = sqrt(e1);
    g->el[2] = sqrt(e2);
}

static void to_global(const elem_geom *g, double x, double y, double out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = g->v0[d] + g->j[d][0] * x + g->j[d][1] * y;
}

/* Scalar shape functions (shapesets.py:46-70): DP0 -> 1; P1 -> (1-x-y, x, y). */
static void shape_scalar(int nshape, double x, double y, double out[3]) {
    if (nshape == 1) {
        out[0] = 1.0;
    } else {
        out[0] = 1.0 - x - y;
        out[1] = x;
        out[2] = y;
    }
}

/* Piola-mapped RWG reference functions (get_piola_transform :96-111 with the
   rwg0 values of shapesets.py:95-102): J (x, y-1) / |J|, J (x-1, y) / |J|, J (x, y) / |J|. */
static void shape_rwg(const elem_geom *g, double x, double y, double out[3][3]) {
    double r[3][2] = {{x, y - 1.0}, {x - 1.0, y}, {x, y}};
    for (int i = 0; i < 3; ++i)
        for (int d = 0; d < 3; ++d) out[i][d] = (g->j[d][0] * r[i][0] + g->j[d][1] * r[i][1]) / g->ie;
}

/* Kernel functions (numba_kernels.py:176-551).  x = test point, y = trial
   point, nx / ny = test / trial normals, p = kernel parameters. */
static double complex kernel_value(int kernel, const double x[3], const double y[3], const double nx[3],
                                   const double ny[3], const double *p) {
    double diff[3], dist2 = 0.0;
    for (int d = 0; d < 3; ++d) {
        diff[d] = y[d] - x[d];
        dist2 += diff[d] * diff[d];
    }
    double dist = sqrt(dist2);
    switch (kernel) {
    case ORC_LAPLACE_SLP: /* :176 */
        return M_INV_4PI_D / dist;
    case ORC_LAPLACE_DLP: { /* :191, (y - x) . n_y */
        double dot = diff[0] * ny[0] + diff[1] * ny[1] + diff[2] * ny[2];
        return -dot * M_INV_4PI_D / (dist * dist * dist);
    }
    case ORC_LAPLACE_ADLP: { /* :214, (y - x) . n_x */
        double dot = diff[0] * nx[0] + diff[1] * nx[1] + diff[2] * nx[2];
        return dot * M_INV_4PI_D / (dist * dist * dist);
    }
    case ORC_HELMHOLTZ_SLP: { /* :298 */
        double kr = p[0], ki = p[1];
        double complex v = (cos(kr * dist) + I * sin(kr * dist)) * M_INV_4PI_D / dist;
        if (ki != 0.0) v *= exp(-ki * dist);
        return v;
    }
    case ORC_HELMHOLTZ_DLP:
    case ORC_HELMHOLTZ_ADLP: { /* :324 and :363 */
        double kr = p[0], ki = p[1];
        double lg;
        if (kernel == ORC_HELMHOLTZ_DLP)
            lg = (diff[0] * ny[0] + diff[1] * ny[1] + diff[2] * ny[2]);
        else
            lg = -(diff[0] * nx[0] + diff[1] * nx[1] + diff[2] * nx[2]); /* (x - y) . n_x */
        lg *= M_INV_4PI_D / (dist * dist * dist);
        double fr = cos(kr * dist) * lg, fi = sin(kr * dist) * lg;
        if (ki != 0.0) {
            double e = exp(-ki * dist);
            fr *= e;
            fi *= e;
        }
        double a = -1.0 - ki * dist, b = kr * dist;
        return (a * fr - b * fi) + I * (b * fr + a * fi);
    }
    case ORC_HELMHOLTZ_COMBINED: { /* double layer (:324) + eta * single layer (:298), p = (k, eta) */
        double complex dl = kernel_value(ORC_HELMHOLTZ_DLP, x, y, nx, ny, p);
        double complex sl = kernel_value(ORC_HELMHOLTZ_SLP, x, y, nx, ny, p);
        return dl + (p[2] + I * p[3]) * sl;
    }
    case ORC_MODHELM_SLP: /* :443 */
        return M_INV_4PI_D * exp(-p[0] * dist) / dist;
    case ORC_MODHELM_DLP: { /* :479 */
        double dot = diff[0] * ny[0] + diff[1] * ny[1] + diff[2] * ny[2];
        return dot * (-p[0] * dist - 1.0) * M_INV_4PI_D * exp(-p[0] * dist) / (dist * dist * dist);
    }
    case ORC_MODHELM_ADLP: { /* :527 */
        double dot = diff[0] * nx[0] + diff[1] * nx[1] + diff[2] * nx[2];
        return dot * (p[0] * dist + 1.0) * M_INV_4PI_D * exp(-p[0] * dist) / (dist * dist * dist);
    }
    case ORC_FARFIELD_SLP: { /* :402, x is a unit direction */
        double dot = x[0] * y[0] + x[1] * y[1] + x[2] * y[2];
        return M_INV_4PI_D * (cos(-p[0] * dot) + I * sin(-p[0] * dot));
    }
    case ORC_FARFIELD_DLP: { /* :425 */
        double dot = x[0] * y[0] + x[1] * y[1] + x[2] * y[2];
        double factor = -p[0] * (x[0] * ny[0] + x[1] * ny[1] + x[2] * ny[2]);
        return -factor * M_INV_4PI_D * sin(-p[0] * dot) + I * factor * M_INV_4PI_D * cos(-p[0] * dot);
    }
    }
    return 0.0;
}

static int adjacent(const uint32_t *elements, int64_t a, int64_t b) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (elements[i + 3 * a] == elements[j + 3 * b]) return 1;
    return 0;
}

/* Surface curls: row i = n x (jit @ grad_ref[:, i]) * normal_mult, with
   grad_ref = [[-1, 1, 0], [-1, 0, 1]] (numba_kernels.py:1120-1142).  g->n
   already carries the normal multiplier. */
static void surface_curls(const elem_geom *g, double curl[3][3]) {
    static const double gr[2][3] = {{-1.0, 1.0, 0.0}, {-1.0, 0.0, 1.0}};
    for (int i = 0; i < 3; ++i) {
        double sg[3];
        for (int d = 0; d < 3; ++d) sg[d] = g->jit[d][0] * gr[0][i] + g->jit[d][1] * gr[1][i];
        curl[i][0] = g->n[1] * sg[2] - g->n[2] * sg[1];
        curl[i][1] = g->n[2] * sg[0] - g->n[0] * sg[2];
        curl[i][2] = g->n[0] * sg[1] - g->n[1] * sg[0];
    }
}

static void add_result(double *result, int is_complex, int64_t ncols, int64_t row, int64_t col, double complex v) {
    if (is_complex) {
        result[2 * (row * ncols + col)] += creal(v);
        result[2 * (row * ncols + col) + 1] += cimag(v);
    } else {
        result[row * ncols + col] += creal(v);
    }
}

/*
 * Regular-pair dense assembly for one set of test elements (one colour).
 * Follows default_scalar_regular_kernel (:980-1074), laplace_hypersingular_regular
 * (:1078-1200), helmholtz_hypersingular_regular (:1203-1330),
 * modified_helmholtz_hypersingular_regular (:1334-1467),
 * maxwell_efield_regular_assembler (:1853-1970) and
 * maxwell_mfield_regular_assembler (:2151-2278).
 */
int oracle_regular(int assembly, int kernel, const double *params, const double *vertices, int64_t nv,
                   const uint32_t *elements, int64_t ne, int nshape_test, int nshape_trial,
                   const uint32_t *test_elements, int64_t n_test, const uint32_t *trial_elements, int64_t n_trial,
                   const double *test_mult, const double *trial_mult, const uint32_t *test_l2g,
                   const uint32_t *trial_l2g, const int32_t *test_nm, const int32_t *trial_nm,
                   const double *quad_points, const double *quad_weights, int64_t nq, int grids_identical,
                   double *result, int64_t ncols, int is_complex) {
    double complex wavenumber = params[0] + I * params[1];
    int64_t ti;
#pragma omp parallel for schedule(dynamic, 4)
    for (ti = 0; ti < n_test; ++ti) {
        int64_t t = test_elements[ti];
        elem_geom gt;
        geom(vertices, nv, elements, ne, t, (double)test_nm[t], &gt);
        double xt[64][3];
        for (int64_t p = 0; p < nq; ++p) to_global(&gt, quad_points[2 * p], quad_points[2 * p + 1], xt[p]);
        double curl_t[3][3];
        if (assembly >= ORC_ASM_LAPLACE_HYP && assembly <= ORC_ASM_MODHELM_HYP) surface_curls(&gt, curl_t);
        for (int64_t si = 0; si < n_trial; ++si) {
            int64_t s = trial_elements[si];
            if (grids_identical && adjacent(elements, t, s)) continue;
            elem_geom gs;
            geom(vertices, nv, elements, ne, s, (double)trial_nm[s], &gs);
            double complex local[3][3] = {{0}};
            double curl_s[3][3];
            if (assembly >= ORC_ASM_LAPLACE_HYP && assembly <= ORC_ASM_MODHELM_HYP) surface_curls(&gs, curl_s);
            double normal_prod = gt.n[0] * gs.n[0] + gt.n[1] * gs.n[1] + gt.n[2] * gs.n[2];
            for (int64_t p = 0; p < nq; ++p) {
                double phi_t[3];
                shape_scalar(nshape_test, quad_points[2 * p], quad_points[2 * p + 1], phi_t);
                double bt[3][3] = {{0}};
                if (assembly >= ORC_ASM_EFIE) shape_rwg(&gt, quad_points[2 * p], quad_points[2 * p + 1], bt);
                for (int64_t q = 0; q < nq; ++q) {
                    double ys[3];
                    to_global(&gs, quad_points[2 * q], quad_points[2 * q + 1], ys);
                    double complex kv = kernel_value(kernel, xt[p], ys, gt.n, gs.n, params);
                    double complex tmp = kv * (quad_weights[q] * gs.ie * gt.ie * quad_weights[p]);
                    double phi_s[3];
                    shape_scalar(nshape_trial, quad_points[2 * q], quad_points[2 * q + 1], phi_s);
                    if (assembly == ORC_ASM_SCALAR) {
                        for (int i = 0; i < nshape_test; ++i)
                            for (int j = 0; j < nshape_trial; ++j) local[i][j] += tmp * phi_s[j] * phi_t[i];
                    } else if (assembly == ORC_ASM_LAPLACE_HYP || assembly == ORC_ASM_HELM_HYP ||
                               assembly == ORC_ASM_MODHELM_HYP) {
                        double complex k2 = (assembly == ORC_ASM_HELM_HYP) ? -wavenumber * wavenumber
                                            : (assembly == ORC_ASM_MODHELM_HYP) ? params[0] * params[0]
                                                                                : 0.0;
                        for (int i = 0; i < 3; ++i)
                            for (int j = 0; j < 3; ++j) {
                                double cp = curl_t[i][0] * curl_s[j][0] + curl_t[i][1] * curl_s[j][1] +
                                            curl_t[i][2] * curl_s[j][2];
                                local[i][j] += tmp * (cp + k2 * phi_t[i] * phi_s[j] * normal_prod);
                            }
                    } else {
                        double bs[3][3];
                        shape_rwg(&gs, quad_points[2 * q], quad_points[2 * q + 1], bs);
                        if (assembly == ORC_ASM_EFIE) {
                            double div = 4.0 / (gt.ie * gs.ie);
                            for (int i = 0; i < 3; ++i)
                                for (int j = 0; j < 3; ++j) {
                                    double dot = bt[i][0] * bs[j][0] + bt[i][1] * bs[j][1] + bt[i][2] * bs[j][2];
                                    local[i][j] += tmp * (-I * wavenumber * dot - div / (I * wavenumber));
                                }
                        } else {
                            double diff[3] = {xt[p][0] - ys[0], xt[p][1] - ys[1], xt[p][2] - ys[2]};
                            double dist = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                            double complex f = (I * wavenumber * dist - 1.0) / (dist * dist);
                            for (int i = 0; i < 3; ++i)
                                for (int j = 0; j < 3; ++j) {
                                    double c[3] = {bt[i][1] * bs[j][2] - bt[i][2] * bs[j][1],
                                                   bt[i][2] * bs[j][0] - bt[i][0] * bs[j][2],
                                                   bt[i][0] * bs[j][1] - bt[i][1] * bs[j][0]};
                                    local[i][j] += tmp * (diff[0] * c[0] + diff[1] * c[1] + diff[2] * c[2]) * f;
                                }
                        }
                    }
                }
            }
            for (int i = 0; i < nshape_test; ++i)
                for (int j = 0; j < nshape_trial; ++j) {
                    double complex v =
                        local[i][j] * test_mult[t * nshape_test + i] * trial_mult[s * nshape_trial + j];
                    if (assembly >= ORC_ASM_EFIE) v *= gt.el[i] * gs.el[j];
                    add_result(result, is_complex, ncols, test_l2g[t * nshape_test + i],
                               trial_l2g[s * nshape_trial + j], v);
                }
        }
    }
    return 0;
}

/*
 * Singular pairs (default_scalar_singular_kernel :1471-1526,
 * laplace_hypersingular_singular :1530-1608, helmholtz_hypersingular_singular
 * :1612-1694, modified_helmholtz_hypersingular_singular :1698-1784,
 * maxwell_efield_singular :1973-2061, maxwell_mfield_singular :2065-2147).
 * result: flat (npairs * nshape_test * nshape_trial), accumulated into.
 * test_points / trial_points: (2, P) Fortran order, i.e. pts[2 * k + c].
 */
int oracle_singular(int assembly, int kernel, const double *params, const double *vertices, int64_t nv,
                    const uint32_t *elements, int64_t ne, int nshape_test, int nshape_trial,
                    const double *test_points, const double *trial_points, const double *weights,
                    const uint32_t *test_elems, const uint32_t *trial_elems, const uint32_t *test_off,
                    const uint32_t *trial_off, const uint32_t *weights_off, const uint32_t *npoints,
                    int64_t npairs, const int32_t *test_nm, const int32_t *trial_nm, double *result,
                    int is_complex) {
    double complex wavenumber = params[0] + I * params[1];
    int64_t k;
#pragma omp parallel for schedule(dynamic, 8)
    for (k = 0; k < npairs; ++k) {
        int64_t t = test_elems[k], s = trial_elems[k];
        elem_geom gt, gs;
        geom(vertices, nv, elements, ne, t, (double)test_nm[t], &gt);
        geom(vertices, nv, elements, ne, s, (double)trial_nm[s], &gs);
        double curl_t[3][3], curl_s[3][3];
        surface_curls(&gt, curl_t);
        surface_curls(&gs, curl_s);
        double normal_prod = gt.n[0] * gs.n[0] + gt.n[1] * gs.n[1] + gt.n[2] * gs.n[2];
        double complex acc[3][3] = {{0}};
        for (uint32_t m = 0; m < npoints[k]; ++m) {
            const double *tp = test_points + 2 * (int64_t)(test_off[k] + m);
            const double *sp = trial_points + 2 * (int64_t)(trial_off[k] + m);
            double w = weights[weights_off[k] + m];
            double x[3], y[3];
            to_global(&gt, tp[0], tp[1], x);
            to_global(&gs, sp[0], sp[1], y);
            double complex kv = kernel_value(kernel, x, y, gt.n, gs.n, params);
            double pt[3], ps[3];
            shape_scalar(nshape_test, tp[0], tp[1], pt);
            shape_scalar(nshape_trial, sp[0], sp[1], ps);
            if (assembly == ORC_ASM_SCALAR) {
                for (int i = 0; i < nshape_test; ++i)
                    for (int j = 0; j < nshape_trial; ++j) acc[i][j] += kv * w * pt[i] * ps[j];
            } else if (assembly == ORC_ASM_LAPLACE_HYP) {
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) acc[i][j] += kv * w;
            } else if (assembly == ORC_ASM_HELM_HYP || assembly == ORC_ASM_MODHELM_HYP) {
                double complex k2 = (assembly == ORC_ASM_HELM_HYP) ? -wavenumber * wavenumber : params[0] * params[0];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        double cp = curl_t[i][0] * curl_s[j][0] + curl_t[i][1] * curl_s[j][1] +
                                    curl_t[i][2] * curl_s[j][2];
                        acc[i][j] += kv * (cp + k2 * pt[i] * ps[j] * normal_prod) * w;
                    }
            } else {
                double bt[3][3], bs[3][3];
                shape_rwg(&gt, tp[0], tp[1], bt);
                shape_rwg(&gs, sp[0], sp[1], bs);
                if (assembly == ORC_ASM_EFIE) {
                    double complex div = 4.0 / (I * wavenumber * gt.ie * gs.ie);
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            double dot = bt[i][0] * bs[j][0] + bt[i][1] * bs[j][1] + bt[i][2] * bs[j][2];
                            acc[i][j] += kv * (-I * wavenumber * dot - div) * w * gt.el[i] * gs.el[j];
                        }
                } else {
                    double diff[3] = {x[0] - y[0], x[1] - y[1], x[2] - y[2]};
                    double dist = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                    double complex f = (I * wavenumber * dist - 1.0) / (dist * dist);
                    for (int i = 0; i < 3; ++i)
                        for (int j = 0; j < 3; ++j) {
                            double c[3] = {bt[i][1] * bs[j][2] - bt[i][2] * bs[j][1],
                                           bt[i][2] * bs[j][0] - bt[i][0] * bs[j][2],
                                           bt[i][0] * bs[j][1] - bt[i][1] * bs[j][0]};
                            acc[i][j] += kv * f * (diff[0] * c[0] + diff[1] * c[1] + diff[2] * c[2]) * w *
                                         gt.el[i] * gs.el[j];
                        }
                }
            }
        }
        for (int i = 0; i < nshape_test; ++i)
            for (int j = 0; j < nshape_trial; ++j) {
                double complex v = acc[i][j] * (gt.ie * gs.ie);
                if (assembly == ORC_ASM_LAPLACE_HYP) {
                    double cp = curl_t[i][0] * curl_s[j][0] + curl_t[i][1] * curl_s[j][1] + curl_t[i][2] * curl_s[j][2];
                    v *= cp;
                }
                int64_t idx = (int64_t)nshape_trial * nshape_test * k + i * nshape_trial + j;
                if (is_complex) {
                    result[2 * idx] += creal(v);
                    result[2 * idx + 1] += cimag(v);
                } else {
                    result[idx] += creal(v);
                }
            }
    }
    return 0;
}

/*
 * Potential evaluation (default_scalar_potential_kernel :1788-1849,
 * maxwell_efield_potential :2281-2359, maxwell_mfield_potential :2363-2433,
 * maxwell_efield_far_field :2437-2503, maxwell_mfield_far_field :2507-2570).
 * assembly: 0 scalar, 4 electric, 5 magnetic; kernel selects the Green's
 * function (far-field kernels treat the points as directions).
 * points: (3, P) Fortran order; x: complex localised coefficients
 * (nshape * ne) interleaved; result: (kdim, P) complex, row-major.
 */
int oracle_potential(int assembly, int kernel, const double *params, const double *vertices, int64_t nv,
                     const uint32_t *elements, int64_t ne, int nshape, const uint32_t *support, int64_t nsupport,
                     const int32_t *nm, const double *quad_points, const double *quad_weights, int64_t nq,
                     const double *points, int64_t npoints, const double *x, double *result) {
    double complex wavenumber = params[0] + I * params[1];
    int64_t nsrc = nsupport * nq;
    double *src = (double *)malloc(sizeof(double) * 6 * nsrc);          /* point + normal */
    double complex *tmp = (double complex *)malloc(sizeof(double complex) * 4 * nsrc); /* scalar or 3-vector + div */
    for (int64_t ei = 0; ei < nsupport; ++ei) {
        int64_t e = support[ei];
        elem_geom g;
        geom(vertices, nv, elements, ne, e, (double)nm[e], &g);
        for (int64_t q = 0; q < nq; ++q) {
            int64_t k = ei * nq + q;
            to_global(&g, quad_points[2 * q], quad_points[2 * q + 1], src + 6 * k);
            for (int d = 0; d < 3; ++d) src[6 * k + 3 + d] = g.n[d];
            const double *xe = x + 2 * nshape * e;
            if (assembly == ORC_ASM_SCALAR) {
                double phi[3];
                shape_scalar(nshape, quad_points[2 * q], quad_points[2 * q + 1], phi);
                double complex acc = 0.0;
                for (int i = 0; i < nshape; ++i)
                    acc += g.ie * quad_weights[q] * phi[i] * (xe[2 * i] + I * xe[2 * i + 1]);
                tmp[4 * k] = acc;
            } else {
                double b[3][3];
                shape_rwg(&g, quad_points[2 * q], quad_points[2 * q + 1], b);
                double complex v[3] = {0, 0, 0}, dv = 0.0;
                for (int i = 0; i < 3; ++i) {
                    double complex factor = quad_weights[q] * (xe[2 * i] + I * xe[2 * i + 1]) * g.el[i];
                    for (int d = 0; d < 3; ++d) v[d] += factor * b[i][d] * g.ie;
                    dv += 2.0 * factor;
                }
                for (int d = 0; d < 3; ++d) tmp[4 * k + d] = v[d];
                tmp[4 * k + 3] = dv;
            }
        }
    }
    int far = (kernel == ORC_FARFIELD_SLP || kernel == ORC_FARFIELD_DLP);
    int kdim = (assembly == ORC_ASM_SCALAR) ? 1 : 3;
    static const double zero[3] = {0.0, 0.0, 0.0};
    int64_t pi;
#pragma omp parallel for schedule(static)
    for (pi = 0; pi < npoints; ++pi) {
        double xp[3] = {points[3 * pi], points[3 * pi + 1], points[3 * pi + 2]};
        double complex acc[3] = {0, 0, 0};
        for (int64_t k = 0; k < nsrc; ++k) {
            const double *y = src + 6 * k;
            double complex kv = kernel_value(kernel, xp, y, zero, y + 3, params);
            if (assembly == ORC_ASM_SCALAR) {
                acc[0] += kv * tmp[4 * k];
            } else if (far) {
                if (assembly == ORC_ASM_EFIE) {
                    for (int d = 0; d < 3; ++d) acc[d] += kv * (I * wavenumber * tmp[4 * k + d] - xp[d] * tmp[4 * k + 3]);
                } else {
                    double complex val[3];
                    for (int d = 0; d < 3; ++d) val[d] = kv * I * wavenumber * tmp[4 * k + d];
                    acc[0] += xp[1] * val[2] - xp[2] * val[1];
                    acc[1] += xp[2] * val[0] - xp[0] * val[2];
                    acc[2] += xp[0] * val[1] - xp[1] * val[0];
                }
            } else {
                double diff[3] = {xp[0] - y[0], xp[1] - y[1], xp[2] - y[2]};
                double dist = sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
                if (assembly == ORC_ASM_EFIE) {
                    for (int d = 0; d < 3; ++d)
                        acc[d] += kv * (I * wavenumber * tmp[4 * k + d] -
                                        diff[d] * (I * wavenumber * dist - 1.0) * tmp[4 * k + 3] /
                                            (I * wavenumber * dist * dist));
                } else {
                    double complex val[3];
                    for (int d = 0; d < 3; ++d) val[d] = kv * (I * wavenumber * dist - 1.0) * tmp[4 * k + d] / (dist * dist);
                    acc[0] += diff[1] * val[2] - diff[2] * val[1];
                    acc[1] += diff[2] * val[0] - diff[0] * val[2];
                    acc[2] += diff[0] * val[1] - diff[1] * val[0];
                }
            }
        }
        for (int d = 0; d < kdim; ++d) {
            result[2 * (d * npoints + pi)] = creal(acc[d]);
            result[2 * (d * npoints + pi) + 1] = cimag(acc[d]);
        }
    }
    free(src);
    free(tmp);
    return 0;
}
