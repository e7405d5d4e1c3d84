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
    from bempp_cuda.grid_function import project_callable
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
