"""Grid functions: coefficients in a space and projections onto a dual space.

Mirrors the parts of ``bempp_cl.api.assembly.grid_function.GridFunction``
(grid_function.py:127-330, 428-453) that the dense solve path uses:
construction from coefficients, projections or a callable, and
``projections(dual_space)``.  A callable is projected with the regular
triangle rule exactly as ``_project_function_vectorized`` does
(grid_function.py:824-863): sum over quadrature points of
w_q * phi_i(q) * f(x_q) * |J|.

Callables are vectorized numpy functions ``fun(x, n, domain_index, result)``
with x, n of shape (3, npoints), domain_index (npoints,) and result
(codomain_dimension, npoints) filled in place (the reference's vectorized
callable convention).
"""

import numpy as _np

from .quadrature import triangle_rule


def _local_values(space, points):
    """Shape values (codomain, nshape, npoints) on every support element."""
    return space.shapeset.evaluate(points)


class GridFunction(object):
    def __init__(self, space, dual_space=None, fun=None, coefficients=None, projections=None, parameters=None,
                 complex=True):
        if sum(v is not None for v in (fun, coefficients, projections)) != 1:
            raise ValueError("Exactly one of fun, coefficients and projections must be given.")
        if space.codomain_dimension != 1 and fun is not None:
            raise ValueError("callable projection is implemented for scalar spaces")
        self.space = space
        self.dual_space = dual_space if dual_space is not None else space
        self._coefficients = None if coefficients is None else _np.asarray(coefficients)
        self._projections = None if projections is None else _np.asarray(projections)
        order = parameters.quadrature.regular if parameters is not None else 4
        if fun is not None:
            self._projections = project_callable(fun, self.dual_space, order, complex)

    @property
    def coefficients(self):
        if self._coefficients is None:
            if self.space.number_of_shape_functions != 1 or not (self.space == self.dual_space):
                raise ValueError("coefficients from projections are implemented for identical DP0 spaces")
            areas = _np.asarray(self.space.grid.volumes)[self.space.support_elements]
            self._coefficients = self._projections / areas
        return self._coefficients

    def projections(self, dual_space=None):
        dual_space = self.dual_space if dual_space is None else dual_space
        if self._projections is not None and dual_space == self.dual_space:
            return self._projections
        if self.space.number_of_shape_functions == 1 and dual_space.number_of_shape_functions == 1 and (
            self.space == dual_space
        ):
            areas = _np.asarray(self.space.grid.volumes)[self.space.support_elements]
            return areas * self.coefficients
        raise ValueError("projections onto a different space are implemented for identical DP0 spaces")


def project_callable(fun, dual_space, order=4, complex=True):
    """Vector of projections <fun, phi_i> onto ``dual_space`` (grid_function.py:824-863)."""
    grid = dual_space.grid
    points, weights = triangle_rule(order)
    sup = _np.asarray(dual_space.support_elements, dtype=_np.int64)
    e = grid.elements.astype(_np.int64)[:, sup]
    v = grid.vertices
    b0 = 1.0 - points[0] - points[1]
    # global points (3, nsup, nq) as barycentric combinations of the corners
    gp = (v[:, e[0]][:, :, None] * b0 + v[:, e[1]][:, :, None] * points[0] + v[:, e[2]][:, :, None] * points[1])
    nq = len(weights)
    normals = (grid.normals[sup] * dual_space.normal_multipliers[sup][:, None]).T
    x = gp.reshape(3, -1)
    n = _np.repeat(normals, nq, axis=1)
    dom = _np.repeat(grid.domain_indices[sup], nq)
    values = _np.zeros((1, x.shape[1]), dtype=_np.complex128 if complex else _np.float64)
    fun(x, n, dom, values)
    values = values.reshape(len(sup), nq)
    shape = _local_values(dual_space, points)[0]  # (nshape, nq)
    ie = grid.integration_elements[sup]
    local = _np.einsum("eq,iq,q->ei", values, shape, weights) * ie[:, None]
    out = _np.zeros(dual_space.global_dof_count, dtype=values.dtype)
    l2g = dual_space.local2global[sup]
    mult = dual_space.local_multipliers[sup]
    _np.add.at(out, l2g.ravel(), (local * mult).ravel())
    return out
