"""Host (oracle) evaluation of the far-field scattering objective.

Test infrastructure: restates, with the C oracle's assembly and potential
kernels and numpy, the forward map that bempp_cuda.shape_gradient evaluates
on the device, so the GPU objective and its adjoint gradient can be checked
against central differences of an independent implementation.

    A = DLP - 1/2 I - i k SLP (DP0),  b = projection of -exp(i k d_inc . x)
    phi = A^-1 b,  u = (DLP_ff - i k SLP_ff) phi,  J = sum |u|^2
"""

import numpy as np


def host_objective(vertices, elements, k, directions, incident=(0.0, 0.0, 1.0)):
    """J for vertices (nv, 3) and elements (ne, 3), all on the host."""
    from bempp_cuda.grid import Grid
    from bempp_cuda.quadrature import SingularPairs, triangle_rule
    from bempp_cuda.space import function_space

    from oracle import oracle as orc

    grid = Grid(np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).T),
                np.ascontiguousarray(np.asarray(elements).T))
    space = function_space(grid, "DP", 0)
    qp, qw = triangle_rule(4)
    rule = SingularPairs(grid, 4, space.support, space.support).arrays()
    a = orc.assemble_dense("helmholtz_combined_field", "default_scalar", [k, 0.0, 0.0, -k], True, space, space, qp,
                           qw, rule)
    a[np.diag_indices_from(a)] -= 0.25 * grid.integration_elements
    d = np.asarray(incident, dtype=np.float64)

    def minus_incident(x, n, domain_index, result):
        result[0] = -np.exp(1j * k * (d @ x))

    b = project_callable(minus_incident, space, 4, True)
    phi = np.linalg.solve(a, b)
    dirs = np.ascontiguousarray(np.asarray(directions, dtype=np.float64).T)
    dlp = orc.evaluate_potential("helmholtz_far_field_double_layer", "default_scalar", [k], space, dirs, phi, qp, qw)
    slp = orc.evaluate_potential("helmholtz_far_field_single_layer", "default_scalar", [k], space, dirs, phi, qp, qw)
    u = dlp[0] - 1j * k * slp[0]
    return float(np.sum(np.abs(u) ** 2)), a, b, u


def project_callable(fun, dual_space, order=4, complex=True):
    """Host restatement of the reference's vectorized projection (grid_function.py:824-863): the
    check of bempp_cuda.grid_function.project_callable_device."""
    from bempp_cuda.quadrature import triangle_rule

    grid = dual_space.grid
    points, weights = triangle_rule(order)
    sup = np.asarray(dual_space.support_elements, dtype=np.int64)
    e = grid.elements.astype(np.int64)[:, sup]
    v = grid.vertices
    b0 = 1.0 - points[0] - points[1]
    # global points (3, nsup, nq) as barycentric combinations of the corners
    gp = (v[:, e[0]][:, :, None] * b0 + v[:, e[1]][:, :, None] * points[0] + v[:, e[2]][:, :, None] * points[1])
    nq = len(weights)
    normals = (grid.normals[sup] * dual_space.normal_multipliers[sup][:, None]).T
    x = gp.reshape(3, -1)
    n = np.repeat(normals, nq, axis=1)
    dom = np.repeat(grid.domain_indices[sup], nq)
    values = np.zeros((1, x.shape[1]), dtype=np.complex128 if complex else np.float64)
    fun(x, n, dom, values)
    values = values.reshape(len(sup), nq)
    shape = dual_space.shapeset.evaluate(points)[0]  # (nshape, nq)
    ie = grid.integration_elements[sup]
    local = np.einsum("eq,iq,q->ei", values, shape, weights) * ie[:, None]
    out = np.zeros(dual_space.global_dof_count, dtype=values.dtype)
    l2g = dual_space.local2global[sup]
    mult = dual_space.local_multipliers[sup]
    np.add.at(out, l2g.ravel(), (local * mult).ravel())
    return out
