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
callable convention), or functions marked with ``device_callable``, which
take the same arguments as CUDA tensors and return the values (npoints,) as
a tensor.  Both go through the device kernels (``bemppcuda_quadrature_points``,
``bemppcuda_project``): the points and normals of the rule are formed on the
device, a device callable is evaluated there (the whole projection stays in
HBM), a host callable on copies of them; the weighted sums and the scatter
onto the dofs run on the device.
"""

import numpy as _np


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
            proj = project_callable_device(fun, self.dual_space, order)
            self._projections = proj.cpu().numpy() if complex else proj.real.cpu().numpy()

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


def device_callable(fun):
    """Mark ``fun(x, n, domain_index) -> values`` as a device callable: x, n (3, npoints) float64 and
    domain_index (npoints,) int32 CUDA tensors in, the (npoints,) values (real or complex) out."""
    fun.bempp_cuda_device = True
    return fun


def project_callable_device(fun, dual_space, order=4):
    """Projections <fun, phi_i> onto the scalar ``dual_space`` as a complex128 CUDA tensor
    (grid_function.py, _project_function_vectorized, on the device)."""
    import torch

    from . import _lib
    from .assembly import regular_rule
    from .device import current_stream, device_grid, device_space, ptr, require_cuda

    require_cuda()
    if dual_space.codomain_dimension != 1:
        raise ValueError("callable projection is implemented for scalar spaces")
    grid = dual_space.grid
    dgrid = device_grid(grid)
    dspace = device_space(dual_space)
    qp, qw = regular_rule(order)
    nq = len(qw)
    nsup = dspace.nsupport
    grec, srec = dgrid.record(), dspace.record()
    lib = _lib.load()
    points = torch.empty((3, nsup * nq), dtype=torch.float64, device="cuda")
    normals = torch.empty((3, nsup * nq), dtype=torch.float64, device="cuda")
    _lib.check(lib.bemppcuda_quadrature_points(grec, srec, nq, qp.ctypes.data, qw.ctypes.data, ptr(points),
                                               ptr(normals), current_stream()))
    sup = _np.asarray(dual_space.support_elements, dtype=_np.int64)
    dom = _np.repeat(_np.asarray(grid.domain_indices)[sup], nq).astype(_np.int32)
    if getattr(fun, "bempp_cuda_device", False):
        values = fun(points, normals, torch.as_tensor(dom, device="cuda"))
        values = torch.as_tensor(values, device="cuda").reshape(-1).to(torch.complex128).contiguous()
    else:
        host = _np.zeros((1, nsup * nq), dtype=_np.complex128)
        fun(points.cpu().numpy(), normals.cpu().numpy(), dom, host)
        values = torch.as_tensor(host[0], device="cuda")
    if values.numel() != nsup * nq:
        raise ValueError("the callable returned %d values for %d points" % (values.numel(), nsup * nq))
    out = torch.empty(int(dual_space.global_dof_count), dtype=torch.complex128, device="cuda")
    _lib.check(lib.bemppcuda_project(grec, srec, nq, qp.ctypes.data, qw.ctypes.data, ptr(values), ptr(out),
                                     current_stream()))
    return out
