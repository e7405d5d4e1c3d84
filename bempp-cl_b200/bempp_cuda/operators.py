"""Operator factories mirroring ``bempp_cl.api.operators`` for the cuda interface.

The factories build the same ``OperatorDescriptor`` the reference builds
(bempp_cl/api/operators/__init__.py:11-14; identifiers, option arrays,
kernel and assembly types as in boundary/{laplace,helmholtz,
modified_helmholtz,maxwell}.py, potential/*.py and far_field/*.py), so a
script written against the reference reads the same here:

    space = function_space(grid, "DP", 0)
    op = boundary.helmholtz.single_layer(space, space, space, 10.0)
    mat = op.weak_form()          # DenseDeviceOperator, matrix in HBM
    y = mat @ x                    # device matvec

This module exists so the path can run where bempp_cl is not installed; when
it is, ``bempp_cuda.plugin.install()`` makes the reference's own factories
accept ``device_interface="cuda"`` instead.
"""

import collections as _collections
import types as _types

import numpy as _np
import torch as _torch

OperatorDescriptor = _collections.namedtuple(
    "OperatorDescriptor",
    "identifier options kernel_type assembly_type precision is_complex singular_part kernel_dimension",
)


class _Quadrature(object):
    def __init__(self):
        self.regular = 4
        self.singular = 4


class Parameters(object):
    """Quadrature orders read by the assembly (api/utils/parameters.py:27-28)."""

    def __init__(self):
        self.quadrature = _Quadrature()


def _params(parameters):
    return parameters if parameters is not None else Parameters()


class DenseDeviceOperator(object):
    """Dense discrete operator whose matrix stays on the GPU.

    Mirrors DenseDiscreteBoundaryOperator (discrete_boundary_operator.py:177-252):
    ``shape``, ``dtype``, ``A`` (host copy), ``@`` / ``dot`` (device matvec /
    matmat for device tensors, host in -> host out for ndarrays) and linear
    combinations.
    """

    def __init__(self, tensor):
        self.tensor = tensor

    @property
    def shape(self):
        return tuple(self.tensor.shape)

    @property
    def dtype(self):
        return _np.complex128 if self.tensor.is_complex() else _np.float64

    @property
    def A(self):
        return self.tensor.cpu().numpy()

    def to_dense(self):
        return self.A

    def dot(self, x):
        if isinstance(x, _torch.Tensor):
            xt = x.to(self.tensor.dtype) if not self.tensor.is_complex() or x.is_complex() else x.to(self.tensor.dtype)
            if xt.dim() == 1 and self.tensor.is_cuda and self.tensor.is_complex() and self.tensor.stride(1) == 1:
                from .matmat import gemv

                return gemv(self.tensor, xt)
            return self.tensor @ xt
        x = _np.asarray(x)
        cdtype = _torch.complex128 if (self.tensor.is_complex() or _np.iscomplexobj(x)) else _torch.float64
        mat = self.tensor if self.tensor.dtype == cdtype else self.tensor.to(cdtype)
        return (mat @ _torch.as_tensor(x).to(device=self.tensor.device, dtype=cdtype)).cpu().numpy()

    def __matmul__(self, x):
        return self.dot(x)

    def __call__(self, x):
        return self.dot(x)

    def _combine(self, other, a, b):
        if isinstance(other, DenseDeviceOperator):
            t1, t2 = self.tensor, other.tensor
            if t1.is_complex() != t2.is_complex():
                t1, t2 = t1.to(_torch.complex128), t2.to(_torch.complex128)
            return DenseDeviceOperator(a * t1 + b * t2)
        if isinstance(other, DiagonalOperator):
            out = self.tensor * a if a != 1 else self.tensor.clone()
            vals = other.values.to(out.device)
            if not out.is_complex() and (vals.is_complex() or isinstance(b, complex)):
                out = out.to(_torch.complex128)
            out.diagonal().add_(b * vals.to(out.dtype))
            return DenseDeviceOperator(out)
        if isinstance(other, SparseDeviceOperator):
            out = self.tensor * a if a != 1 else self.tensor.clone()
            if not out.is_complex() and (other._coo.is_complex() or isinstance(b, complex)):
                out = out.to(_torch.complex128)
            other.add_into(out, b)
            return DenseDeviceOperator(out)
        return NotImplemented

    def __add__(self, other):
        return self._combine(other, 1, 1)

    def __radd__(self, other):
        return self.__add__(other)

    def __sub__(self, other):
        return self._combine(other, 1, -1)

    def __mul__(self, alpha):
        if _np.isscalar(alpha):
            t = self.tensor
            if isinstance(alpha, complex) and not t.is_complex():
                t = t.to(_torch.complex128)
            return DenseDeviceOperator(t * alpha)
        return self.dot(alpha)

    def __rmul__(self, alpha):
        return self.__mul__(alpha)

    def __neg__(self):
        return DenseDeviceOperator(-self.tensor)


class DiagonalOperator(object):
    """Diagonal discrete operator (the DP0 mass matrix) with device values."""

    def __init__(self, values):
        self.values = values

    @property
    def shape(self):
        n = self.values.shape[0]
        return (n, n)

    def __mul__(self, alpha):
        return DiagonalOperator(self.values * alpha)

    __rmul__ = __mul__

    def __neg__(self):
        return DiagonalOperator(-self.values)


class SparseDeviceOperator(object):
    """Sparse discrete operator on the device: the counterpart of SparseDiscreteBoundaryOperator
    (discrete_boundary_operator.py:255-330) with coalesced COO triplets and a CSR copy for products."""

    def __init__(self, rows, cols, values, shape):
        coo = _torch.sparse_coo_tensor(_torch.stack([rows, cols]), values, size=tuple(shape)).coalesce()
        self._coo = coo
        self.tensor = coo.to_sparse_csr()

    @property
    def shape(self):
        return tuple(self._coo.shape)

    @property
    def dtype(self):
        return _np.complex128 if self._coo.is_complex() else _np.float64

    @property
    def A(self):
        return self._coo.to_dense().cpu().numpy()

    def to_dense(self):
        return self.A

    def add_into(self, dense, coef=1.0):
        """dense += coef * self, scattered on the device."""
        idx = self._coo.indices()
        vals = self._coo.values() * coef
        if vals.is_complex() and not dense.is_complex():
            raise TypeError("a complex sparse term needs a complex dense operator")
        dense.index_put_((idx[0], idx[1]), vals.to(dense.dtype), accumulate=True)
        return dense

    def dot(self, x):
        host = not isinstance(x, _torch.Tensor)
        xt = _torch.as_tensor(_np.asarray(x)).to("cuda") if host else x
        mat = self.tensor
        if xt.is_complex() and not mat.is_complex():
            mat = mat.to(xt.dtype)
        elif mat.is_complex() and not xt.is_complex():
            xt = xt.to(mat.dtype)
        y = mat @ xt.to(mat.dtype)
        return y.cpu().numpy() if host else y

    def __matmul__(self, x):
        return self.dot(x)

    def __call__(self, x):
        return self.dot(x)

    def _scaled(self, alpha):
        idx = self._coo.indices()
        return SparseDeviceOperator(idx[0], idx[1], self._coo.values() * alpha, self.shape)

    def __mul__(self, alpha):
        if _np.isscalar(alpha):
            return self._scaled(alpha)
        return self.dot(alpha)

    __rmul__ = __mul__

    def __neg__(self):
        return self._scaled(-1.0)

    def _combine(self, other, a, b):
        if isinstance(other, SparseDeviceOperator):
            i1, i2 = self._coo.indices(), other._coo.indices()
            v1, v2 = self._coo.values() * a, other._coo.values() * b
            if v1.is_complex() != v2.is_complex():
                v1, v2 = v1.to(_torch.complex128), v2.to(_torch.complex128)
            idx = _torch.cat([i1, i2], dim=1)
            return SparseDeviceOperator(idx[0], idx[1], _torch.cat([v1, v2]), self.shape)
        if isinstance(other, DenseDeviceOperator):
            return other._combine(self, b, a)
        return NotImplemented

    def __add__(self, other):
        return self._combine(other, 1, 1)

    def __sub__(self, other):
        return self._combine(other, 1, -1)


class BoundaryOperator(object):
    """Boundary operator with a lazily assembled, cached weak form (boundary_operator.py:36-41)."""

    def __init__(self, domain, range_, dual_to_range, descriptor, device_interface="cuda", parameters=None):
        self.domain = domain
        self.range = range_
        self.dual_to_range = dual_to_range
        self.descriptor = descriptor
        self.device_interface = device_interface or "cuda"
        self.parameters = _params(parameters)
        self._weak_form = None

    def weak_form(self):
        if self._weak_form is None:
            self._weak_form = self._assemble()
        return self._weak_form

    def _assemble(self):
        from .assembly import assemble_dense_device

        return DenseDeviceOperator(
            assemble_dense_device(self.domain, self.dual_to_range, self.parameters, self.descriptor, self.device_interface)
        )

    def __add__(self, other):
        return _SumOperator(self, other, 1.0, 1.0)

    def __sub__(self, other):
        return _SumOperator(self, other, 1.0, -1.0)

    def __mul__(self, alpha):
        return _ScaledOperator(self, alpha)

    __rmul__ = __mul__

    def __neg__(self):
        return _ScaledOperator(self, -1.0)


def linear_terms(op, coef=1.0):
    """Flatten sums and scalings into [(coefficient, leaf operator)]."""
    if isinstance(op, _SumOperator):
        return linear_terms(op._a, coef * op._ca) + linear_terms(op._b, coef * op._cb)
    if isinstance(op, _ScaledOperator):
        return linear_terms(op._op, coef * op._alpha)
    return [(coef, op)]


def _combined_field_parts(op):
    """(a, eta, shift, dlp term) when ``op`` is a DP0 Helmholtz a*DLP + b*SLP + c*I with
    eta = b / a and a real shift = c / a, else None."""
    terms = linear_terms(op)
    dlp = [(c, t) for c, t in terms if t.descriptor is not None and t.descriptor.kernel_type == "helmholtz_double_layer"]
    slp = [(c, t) for c, t in terms if t.descriptor is not None and t.descriptor.kernel_type == "helmholtz_single_layer"
           and t.descriptor.assembly_type == "default_scalar"]
    ident = [(c, t) for c, t in terms if isinstance(t, IdentityOperator)]
    if len(dlp) != 1 or len(slp) != 1 or len(ident) > 1 or len(dlp) + len(slp) + len(ident) != len(terms):
        return None
    (a, d), (b, s) = dlp[0], slp[0]
    if list(d.descriptor.options) != list(s.descriptor.options) or a == 0:
        return None
    if not (d.domain == s.domain and d.dual_to_range == s.dual_to_range):
        return None
    if d.device_interface != s.device_interface:
        return None
    if d.domain.number_of_shape_functions != 1 or d.dual_to_range.number_of_shape_functions != 1:
        return None
    c = ident[0][0] if ident else 0.0
    if ident and not (ident[0][1].domain == d.domain and ident[0][1].dual_to_range == d.dual_to_range):
        return None
    eta = complex(b) / complex(a)
    shift = complex(c) / complex(a)
    if shift.imag != 0.0:
        return None
    return complex(a), eta, shift.real, d


def _fused_combined_field(op):
    """Assemble a DP0 Helmholtz a*DLP + b*SLP + c*I in one pass, or return None.

    The reference assembles each term and adds the dense weak forms
    (boundary_operator.py:134-169); here the shared kernel work (distance,
    exp(ikr)) is done once per quadrature pair (csrc/regular.cu).
    """
    parts = _combined_field_parts(op)
    if parts is None:
        return None
    from .assembly import assemble_combined_field_device

    a, eta, shift, d = parts
    mat = assemble_combined_field_device(d.domain, d.dual_to_range, d.parameters, d.descriptor.options, eta,
                                         shift, d.device_interface)
    if a != 1.0:
        mat.mul_(a)
    return DenseDeviceOperator(mat)


def fp64_matvec(op, matrix):
    """v -> A v with A the FP64 weak form of ``op``, given ``matrix``, a dense weak form of ``op`` held in
    lower precision (``device_interface="cuda_mixed"``): the adjacent element pairs (singular part and
    identity, FP64 in every precision) are taken from ``matrix`` once, the regular part is evaluated
    on the fly in FP64 by the matrix-free apply (csrc/apply.cu), never stored.

    ``op``: a DP0 Helmholtz combined field a*DLP + b*SLP + c*I, or a Laplace / Helmholtz single,
    double or adjoint double layer, on one DP0 space of one grid.  This is the residual product of
    the refined solve (linalg.solve_refined), whose corrections then converge to the FP64 solution.
    """
    parts = _combined_field_parts(op) if isinstance(op, (_SumOperator, _ScaledOperator)) else None
    if parts is not None:
        a, eta, _, d = parts
        opts = list(_np.asarray(d.descriptor.options, dtype=float)[:2]) + [eta.real, eta.imag]
        desc = OperatorDescriptor("helmholtz_combined_field_boundary", opts, "helmholtz_combined_field",
                                  "default_scalar", "double", True, None, 1)
        leaf = d
    elif getattr(op, "descriptor", None) is not None and not isinstance(op, IdentityOperator):
        a, desc, leaf = 1.0, op.descriptor, op
    else:
        raise ValueError("fp64_matvec: a DP0 combined field or a single DP0 boundary operator is required")
    tensor = matrix.tensor if isinstance(matrix, DenseDeviceOperator) else matrix
    return fp64_matvec_of(desc, a, leaf.domain, leaf.parameters, tensor)


def fp64_matvec_of(descriptor, coefficient, space, parameters, matrix):
    """``fp64_matvec`` from its parts: v -> S v + coefficient * A_reg v, S the entries of ``matrix`` at
    the adjacent element pairs of the DP0 ``space``, A_reg the regular part of ``descriptor`` on it."""
    from .assembly import adjacent_part, apply_regular

    singular = adjacent_part(matrix, space, space, parameters)

    def matvec(v):
        v = v.to(_torch.complex128)
        y = _torch.zeros(matrix.shape[0], dtype=_torch.complex128, device=v.device)
        apply_regular(y, v, descriptor, space, space, parameters)
        if coefficient != 1.0:
            y.mul_(coefficient)
        return y + _torch.mv(singular, v)

    return matvec


def weak_form_to_host(op, out=None, blocks=16):
    """The dense weak form of ``op`` as a host tensor (pinned unless ``out`` is given).

    For a DP0 operator of one space (plain, or the fused combined field with
    unit DLP coefficient) the copy to the host overlaps the assembly, one row
    block at a time (assembly.assemble_dense_to_host); otherwise the weak form
    is assembled on the device and copied.  The reference's weak form is a
    host matrix (discrete_boundary_operator.py:177-252), so this is the call
    that hands a user the same object.
    """
    from .assembly import assemble_dense_to_host

    parts = _combined_field_parts(op) if isinstance(op, (_SumOperator, _ScaledOperator)) else None
    if parts is not None and parts[0] == 1.0:
        a, eta, shift, d = parts
        opts = list(_np.asarray(d.descriptor.options, dtype=float)[:2]) + [eta.real, eta.imag]
        desc = OperatorDescriptor("helmholtz_combined_field_boundary", opts, "helmholtz_combined_field",
                                  "default_scalar", "double", True, None, 1)
        return assemble_dense_to_host(d.domain, d.dual_to_range, d.parameters, desc, d.device_interface, out,
                                      diag_shift=shift, blocks=blocks)
    if getattr(op, "descriptor", None) is not None and not isinstance(
            op, (_SumOperator, _ScaledOperator, IdentityOperator)):
        return assemble_dense_to_host(op.domain, op.dual_to_range, op.parameters, op.descriptor,
                                      op.device_interface, out, blocks=blocks)
    w = op.weak_form()
    if isinstance(w, DiagonalOperator):
        t = _torch.diag(w.values)
    elif isinstance(w, SparseDeviceOperator):
        t = w._coo.to_dense()
    else:
        t = w.tensor
    if out is None:
        out = _torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
    out.copy_(t)
    return out


class _SumOperator(BoundaryOperator):
    def __init__(self, a, b, ca, cb):
        super().__init__(a.domain, a.range, a.dual_to_range, None, a.device_interface, a.parameters)
        self._a, self._b, self._ca, self._cb = a, b, ca, cb

    def _assemble(self):
        fused = _fused_combined_field(self)
        if fused is not None:
            return fused
        wa = self._a.weak_form()
        wb = self._b.weak_form()
        if isinstance(wa, (DiagonalOperator, SparseDeviceOperator)) and isinstance(wb, DenseDeviceOperator):
            wa, wb, ca, cb = wb, wa, self._cb, self._ca
        else:
            ca, cb = self._ca, self._cb
        if isinstance(wa, SparseDeviceOperator):
            return wa._combine(wb, ca, cb)
        if isinstance(wb, DiagonalOperator):
            return (wa * ca) + (wb * cb) if ca != 1 else wa + (wb * cb)
        return wa._combine(wb, ca, cb)


class _ScaledOperator(BoundaryOperator):
    def __init__(self, op, alpha):
        super().__init__(op.domain, op.range, op.dual_to_range, None, op.device_interface, op.parameters)
        self._op, self._alpha = op, alpha

    def _assemble(self):
        return self._op.weak_form() * self._alpha


class IdentityOperator(BoundaryOperator):
    """L2 identity (sparse.py:6-28): a diagonal of element areas when domain and dual are the same DP0
    space, else the mass matrix of the two spaces as a device sparse operator (csrc/identity.cu)."""

    def _assemble(self):
        from .assembly import identity_triplets, same_space

        if (self.domain.number_of_shape_functions == 1 and self.dual_to_range.number_of_shape_functions == 1
                and same_space(self.domain, self.dual_to_range) and _dof_is_position(self.domain)):
            areas = _np.asarray(self.domain.grid.volumes)[self.domain.support_elements]
            return DiagonalOperator(_torch.as_tensor(areas, dtype=_torch.float64, device="cuda"))
        rows, cols, values = identity_triplets(self.domain, self.dual_to_range, self.parameters)
        return SparseDeviceOperator(rows, cols, values,
                                    (self.dual_to_range.global_dof_count, self.domain.global_dof_count))


def _dof_is_position(space):
    """DP0 space whose dof i is its i-th support element with multiplier 1 (its mass matrix is diagonal)."""
    l2g = _np.asarray(space.local2global).reshape(-1)
    sup = _np.asarray(space.support_elements)
    mult = _np.asarray(space.local_multipliers).reshape(-1)
    return (len(sup) == int(space.global_dof_count) and _np.array_equal(l2g[sup], _np.arange(len(sup)))
            and bool(_np.all(mult[sup] == 1.0)))


def _create(identifier, domain, range_, dual_to_range, options, kernel_type, assembly_type, is_complex,
            parameters, device_interface, precision):
    descriptor = OperatorDescriptor(
        identifier, list(options), kernel_type, assembly_type, precision or "double", is_complex, None, 1
    )
    return BoundaryOperator(domain, range_, dual_to_range, descriptor, device_interface, parameters)


def _helmholtz_options(k):
    return [float(_np.real(k)), float(_np.imag(k))]


def _boundary(kind, name, kernel_type, assembly_type, is_complex, options_fn):
    def factory(domain, range_, dual_to_range, *args, parameters=None, assembler="dense", device_interface="cuda",
                precision=None):
        options = options_fn(*args)
        return _create(kind + "_" + name + "_boundary", domain, range_, dual_to_range, options, kernel_type,
                       assembly_type, is_complex, parameters, device_interface, precision)

    factory.__name__ = name
    return factory


def _helmholtz_factory(name, kernel, assembly, modified_kernel, modified_assembly):
    def factory(domain, range_, dual_to_range, wavenumber, parameters=None, assembler="dense",
                device_interface="cuda", precision=None):
        if _np.real(wavenumber) == 0:
            # helmholtz.py:22: purely imaginary k -> modified Helmholtz with omega = Im k
            return _create("modified_helmholtz_" + name + "_boundary", domain, range_, dual_to_range,
                           [float(_np.imag(wavenumber))], modified_kernel, modified_assembly, False, parameters,
                           device_interface, precision)
        if name == "hypersingular" and domain.shapeset.identifier != "p1_discontinuous":
            raise ValueError("Domain shapeset must be of type 'p1_discontinuous'.")
        return _create("helmholtz_" + name + "_boundary", domain, range_, dual_to_range,
                       _helmholtz_options(wavenumber), kernel, assembly, True, parameters, device_interface,
                       precision)

    factory.__name__ = name
    return factory


def _maxwell_factory(name, assembly):
    def factory(domain, range_, dual_to_range, wavenumber, parameters=None, assembler="dense",
                device_interface="cuda", precision=None):
        if domain.identifier != "rwg0" or dual_to_range.identifier != "snc0":
            raise ValueError("Operator only defined for domain = 'rwg' and 'dual_to_range = 'snc")
        return _create("maxwell_" + name + "_boundary", domain, range_, dual_to_range, _helmholtz_options(wavenumber),
                       "helmholtz_single_layer", assembly, True, parameters, device_interface, precision)

    factory.__name__ = name
    return factory


def _laplace_hyp(domain, range_, dual_to_range, parameters=None, assembler="dense", device_interface="cuda",
                 precision=None):
    if domain.shapeset.identifier != "p1_discontinuous":
        raise ValueError("Domain shapeset must be of type 'p1_discontinuous'.")
    return _create("laplace_hypersingular_boundary", domain, range_, dual_to_range, [], "laplace_single_layer",
                   "laplace_hypersingular", False, parameters, device_interface, precision)


def _identity(domain, range_, dual_to_range, parameters=None, device_interface="cuda", precision=None):
    descriptor = OperatorDescriptor("l2_identity", [], "l2_identity", "default_sparse", precision or "double",
                                    False, None, 1)
    return IdentityOperator(domain, range_, dual_to_range, descriptor, device_interface, parameters)


boundary = _types.SimpleNamespace(
    laplace=_types.SimpleNamespace(
        single_layer=_boundary("laplace", "single_layer", "laplace_single_layer", "default_scalar", False, lambda: []),
        double_layer=_boundary("laplace", "double_layer", "laplace_double_layer", "default_scalar", False, lambda: []),
        adjoint_double_layer=_boundary("laplace", "adjoint_double_layer", "laplace_adjoint_double_layer",
                                       "default_scalar", False, lambda: []),
        hypersingular=_laplace_hyp,
    ),
    helmholtz=_types.SimpleNamespace(
        single_layer=_helmholtz_factory("single_layer", "helmholtz_single_layer", "default_scalar",
                                        "modified_helmholtz_single_layer", "default_scalar"),
        double_layer=_helmholtz_factory("double_layer", "helmholtz_double_layer", "default_scalar",
                                        "modified_helmholtz_double_layer", "default_scalar"),
        adjoint_double_layer=_helmholtz_factory("adjoint_double_layer", "helmholtz_adjoint_double_layer",
                                                "default_scalar", "modified_helmholtz_adjoint_double_layer",
                                                "default_scalar"),
        hypersingular=_helmholtz_factory("hypersingular", "helmholtz_single_layer", "helmholtz_hypersingular",
                                         "modified_helmholtz_single_layer", "modified_helmholtz_hypersingular"),
    ),
    modified_helmholtz=_types.SimpleNamespace(
        single_layer=_boundary("modified_helmholtz", "single_layer", "modified_helmholtz_single_layer",
                               "default_scalar", False, lambda omega: [float(omega)]),
        double_layer=_boundary("modified_helmholtz", "double_layer", "modified_helmholtz_double_layer",
                               "default_scalar", False, lambda omega: [float(omega)]),
        adjoint_double_layer=_boundary("modified_helmholtz", "adjoint_double_layer",
                                       "modified_helmholtz_adjoint_double_layer", "default_scalar", False,
                                       lambda omega: [float(omega)]),
        hypersingular=_boundary("modified_helmholtz", "hypersingular", "modified_helmholtz_single_layer",
                                "modified_helmholtz_hypersingular", False, lambda omega: [float(omega)]),
    ),
    maxwell=_types.SimpleNamespace(
        electric_field=_maxwell_factory("electric_field", "maxwell_electric_field"),
        magnetic_field=_maxwell_factory("magnetic_field", "maxwell_magnetic_field"),
    ),
    sparse=_types.SimpleNamespace(identity=_identity),
)


class PotentialOperator(object):
    """Potential evaluation operator (potential_operator.py:14; dense_potential_assembler.py:8-40)."""

    def __init__(self, space, points, descriptor, device_interface="cuda", parameters=None):
        self.space = space
        # the operator's own copy: the points are uploaded once per device and reused by every evaluation
        self.points = _np.array(points, dtype=_np.float64, copy=True)
        self.descriptor = descriptor
        self.device_interface = device_interface or "cuda"
        self.parameters = _params(parameters)
        self._points_dev = {}
        self._map_dev = {}

    def _device_points(self):
        """The evaluation points as a (npoints, 3) device tensor on the current device."""
        import torch

        dev = torch.cuda.current_device()
        pts = self._points_dev.get(dev)
        if pts is None:
            pts = torch.as_tensor(_np.ascontiguousarray(self.points.T), device="cuda")
            self._points_dev[dev] = pts
        return pts

    def _device_map(self):
        """``space.map_to_full_grid`` on the current device as a gather: for element-local slot
        e * nshape + i the dof index and its multiplier (index 0 and multiplier 0 outside the support).
        Each slot has one dof, so the gathered product equals the sparse product bit for bit."""
        import torch

        dev = torch.cuda.current_device()
        m = self._map_dev.get(dev)
        if m is None:
            sp = self.space
            nshape = int(sp.number_of_shape_functions)
            ne = int(sp.grid.number_of_elements)
            l2g = _np.asarray(sp.local2global).reshape(-1, nshape)
            mult = _np.asarray(sp.local_multipliers, dtype=_np.float64).reshape(-1, nshape)
            sup = _np.asarray(sp.support_elements, dtype=_np.int64)
            idx = _np.zeros((ne, nshape), dtype=_np.int64)
            mlt = _np.zeros((ne, nshape), dtype=_np.float64)
            idx[sup] = l2g[sup]
            mlt[sup] = mult[sup]
            m = (torch.as_tensor(idx.ravel(), device="cuda"), torch.as_tensor(mlt.ravel(), device="cuda"))
            self._map_dev[dev] = m
        return m

    def evaluate_device(self, coefficients):
        """(kernel_dimension, npoints) complex device tensor for dof ``coefficients`` (host array or
        device tensor of the space's global dof count)."""
        import torch

        from .assembly import evaluate_potential_device, precision_of

        n = int(self.space.global_dof_count)
        if isinstance(coefficients, torch.Tensor):
            coeff = coefficients.to(device="cuda", dtype=torch.complex128).reshape(-1)
        else:
            coeff = torch.as_tensor(_np.ascontiguousarray(_np.asarray(coefficients, dtype=_np.complex128)).reshape(-1),
                                    device="cuda")
        if coeff.shape[0] != n:
            raise ValueError("expected %d coefficients, got %d" % (n, coeff.shape[0]))
        idx, mlt = self._device_map()
        local = coeff.index_select(0, idx) * mlt
        return evaluate_potential_device(self.space, self.descriptor, self._device_points(), local, self.parameters,
                                         precision=precision_of(self.device_interface))

    def evaluate(self, grid_fun):
        coeffs = getattr(grid_fun, "coefficients", grid_fun)
        out = self.evaluate_device(_np.asarray(coeffs, dtype=_np.complex128)).cpu().numpy()
        if not self.descriptor.is_complex and not _np.iscomplexobj(coeffs):
            return out.real.copy()
        return out


def _potential(identifier, kernel_type, assembly_type, is_complex, kdim, options_fn, check=None):
    def factory(space, points, *args, parameters=None, assembler="dense", device_interface="cuda", precision=None):
        if check:
            check(space)
        descriptor = OperatorDescriptor(identifier, list(options_fn(*args)), kernel_type, assembly_type,
                                        precision or "double", is_complex, None, kdim)
        return PotentialOperator(space, points, descriptor, device_interface, parameters)

    return factory


def _require_rwg(space):
    if space.identifier != "rwg0":
        raise ValueError("Space must be an RWG type function space.")


potential = _types.SimpleNamespace(
    laplace=_types.SimpleNamespace(
        single_layer=_potential("laplace_single_layer_potential", "laplace_single_layer", "default_scalar", False, 1,
                                lambda: []),
        double_layer=_potential("laplace_double_layer_potential", "laplace_double_layer", "default_scalar", False, 1,
                                lambda: []),
    ),
    helmholtz=_types.SimpleNamespace(
        single_layer=_potential("helmholtz_single_layer_potential", "helmholtz_single_layer", "default_scalar", True,
                                1, _helmholtz_options),
        double_layer=_potential("helmholtz_double_layer_potential", "helmholtz_double_layer", "default_scalar", True,
                                1, _helmholtz_options),
    ),
    modified_helmholtz=_types.SimpleNamespace(
        single_layer=_potential("modified_helmholtz_single_layer_potential", "modified_helmholtz_single_layer",
                                "default_scalar", False, 1, lambda omega: [float(omega)]),
        double_layer=_potential("modified_helmholtz_double_layer_potential", "modified_helmholtz_double_layer",
                                "default_scalar", False, 1, lambda omega: [float(omega)]),
    ),
    maxwell=_types.SimpleNamespace(
        electric_field=_potential("maxwell_electric_field_potential", "helmholtz_single_layer",
                                  "maxwell_electric_field", True, 3, _helmholtz_options, _require_rwg),
        magnetic_field=_potential("maxwell_magnetic_field_potential", "helmholtz_single_layer",
                                  "maxwell_magnetic_field", True, 3, _helmholtz_options, _require_rwg),
    ),
)

far_field = _types.SimpleNamespace(
    helmholtz=_types.SimpleNamespace(
        single_layer=_potential("helmholtz_far_field_single_layer_potential", "helmholtz_far_field_single_layer",
                                "default_scalar", True, 1, _helmholtz_options),
        double_layer=_potential("helmholtz_far_field_double_layer_potential", "helmholtz_far_field_double_layer",
                                "default_scalar", True, 1, _helmholtz_options),
    ),
    maxwell=_types.SimpleNamespace(
        electric_field=_potential("maxwell_far_field_electric_field_potential", "helmholtz_far_field_single_layer",
                                  "maxwell_electric_far_field", True, 3, _helmholtz_options, _require_rwg),
        magnetic_field=_potential("maxwell_far_field_magnetic_field_potential", "helmholtz_far_field_single_layer",
                                  "maxwell_magnetic_far_field", True, 3, _helmholtz_options, _require_rwg),
    ),
)
