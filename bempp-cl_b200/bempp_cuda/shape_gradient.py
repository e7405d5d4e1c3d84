"""Shape gradient of a far-field scattering objective through an adjoint kernel.

Sound-soft scattering of the plane wave exp(i k d_inc . x) by a closed
surface, indirect combined-field formulation on DP0 (the bempp-cl workflow of
``helmholtz.double_layer - 0.5 * identity - 1j * k * helmholtz.single_layer``,
``GridFunction.projections`` and ``far_field.helmholtz.{double,single}_layer``):

    A phi = b,   A = DLP - 1/2 I - i k SLP,   b = projection of -exp(i k d_inc . x)
    u = F phi,   F = DLP_ff - i k SLP_ff at the unit directions d_j
    J = sum_j |u_j|^2

The gradient with respect to all vertex coordinates and k uses one adjoint
solve, A^H lambda = F^H u, and

    dJ = 2 Re(u^H dF phi) + 2 Re(lambda^H db) - 2 Re(lambda^H dA phi),

evaluated by ``bemppcuda_shape_adjoint_dp0`` (csrc/shape.cu), which recomputes
the quadrature of every element pair instead of forming dA/dx.  The dense
solves run on the device: an LU factorisation (torch.linalg) reused for the
adjoint solve, or GMRES on a complex64 copy of the matrix refined with
complex128 residuals (the adjoint through the transposed view).  The reference has no derivatives; its forward path for this
objective is core/dense_assembler.py:49-98 (operators) and
core/dense_potential_assembler.py:8-40 (far field).
"""

import ctypes as _ct
import math as _math

import numpy as _np
import torch as _torch

from . import _lib
from .assembly import regular_into, regular_rule, singular_into_dense
from .device import current_stream, device_grid, device_singular_rule, device_space, ptr, require_cuda
from .matmat import matvec_of
from .operators import OperatorDescriptor, Parameters
from .space import function_space


def fibonacci_directions(n=32):
    """(n, 3) unit vectors on a Fibonacci (golden-angle) spiral."""
    i = _np.arange(n, dtype=_np.float64) + 0.5
    z = 1.0 - 2.0 * i / n
    rho = _np.sqrt(_np.maximum(0.0, 1.0 - z * z))
    phi = _math.pi * (1.0 + _math.sqrt(5.0)) * i
    return _np.stack([rho * _np.cos(phi), rho * _np.sin(phi), z], axis=1)


class DeviceGeometry(object):
    """Geometry record of a grid whose vertices moved (elements unchanged), built on the device."""

    def __init__(self, base, vertices):
        self.nvertices = base.nvertices
        self.nelements = base.nelements
        self.vertices = vertices.detach().to(dtype=_torch.float64).contiguous()
        if tuple(self.vertices.shape) != (self.nvertices, 3):
            raise ValueError("vertices must have shape (%d, 3)" % self.nvertices)
        self.elements = base.elements
        self.geom = _torch.empty_like(base.geom)
        _lib.check(_lib.load().bemppcuda_grid_geometry(ptr(self.vertices), self.nvertices, ptr(self.elements),
                                                       self.nelements, ptr(self.geom), current_stream()))
        corners = self.vertices[self.elements.long()]
        centroids = corners.mean(dim=1, keepdim=True)
        self.radius = float(((corners - centroids) ** 2).sum(dim=2).sqrt().max().item())

    def record(self):
        return _lib.GridRec(self.nvertices, self.nelements, ptr(self.geom), ptr(self.elements))


class ScatteringState(object):
    """What the backward pass needs from one forward evaluation.

    Holds either the LU factors (``lu``, ``pivots``) or, for the iterative
    solvers, the matrix itself (``matrix``) and its complex64 copy (``low``,
    refined GMRES)."""

    def __init__(self, geometry, lu, pivots, phi, u, farfield, matrix=None, iterations=None, low=None):
        self.geometry = geometry
        self.lu = lu
        self.pivots = pivots
        self.phi = phi
        self.u = u
        self.farfield = farfield
        self.matrix = matrix
        self.iterations = iterations
        self.low = low


class FarFieldObjective(object):
    """J(vertices, k) = sum_j |u_inf(d_j)|^2 for a grid's topology (elements fixed)."""

    def __init__(self, grid, directions=None, incident=(0.0, 0.0, 1.0), parameters=None, solver="lu", tol=1e-12):
        """``solver``: "lu" (dense complex128 LU on the device, factors reused for
        the adjoint solve), "gmres32" (GMRES on a complex64 copy of the matrix,
        refined with complex128 residuals, for both solves), "lu32" (complex64 LU, refined with complex128
        residuals b - A x of the FP64 matrix until ||b - A x|| <= tol ||b||; the
        same factors and refinement for the adjoint) or "gmres" (device GMRES on
        the resident matrix to relative residual ``tol`` for both solves)."""
        require_cuda()
        if solver not in ("lu", "lu32", "gmres", "gmres32"):
            raise ValueError("solver must be 'lu', 'lu32', 'gmres' or 'gmres32'")
        self.solver = solver
        self.tol = float(tol)
        self.grid = grid
        self.parameters = parameters or Parameters()
        if int(self.parameters.quadrature.regular) != 4:
            raise ValueError("the shape gradient uses the 6-point regular rule (order 4)")
        self.space = function_space(grid, "DP", 0)
        self.base = device_grid(grid)
        self.dspace = device_space(self.space)
        if not self.dspace.dof_is_position:
            raise ValueError("the DP0 space must cover every element in order")
        self.rule = device_singular_rule(grid, self.parameters.quadrature.singular, self.space.support,
                                         self.space.support)
        dirs = fibonacci_directions() if directions is None else _np.asarray(directions, dtype=_np.float64)
        self.directions = _torch.as_tensor(_np.ascontiguousarray(dirs), dtype=_torch.float64, device="cuda")
        self.incident = tuple(float(c) for c in incident)
        self.qp, self.qw = regular_rule(4)
        self.workspace = _torch.empty(
            int(_lib.load().bemppcuda_shape_workspace_bytes(self.base.nelements)) // 8, dtype=_torch.float64,
            device="cuda")

    @property
    def vertices(self):
        """Device copy (nv, 3) of the grid's own vertices."""
        return self.base.vertices

    # ------------------------------------------------------------------ pieces of the forward map
    def geometry(self, vertices):
        return DeviceGeometry(self.base, vertices)

    def _args(self, geometry, k):
        a = _lib.ShapeArgs()
        a.grid = geometry.record()
        a.normal_mult = ptr(self.dspace.normal_mult)
        a.k = float(k)
        a.dlp_coeff = 1.0
        a.eta[0], a.eta[1] = 0.0, -float(k)
        a.deta_dk[0], a.deta_dk[1] = 0.0, -1.0
        a.identity = -0.5
        a.nq = len(self.qw)
        a.ndirections = self.directions.shape[0]
        a.quad_points = self.qp.ctypes.data
        a.quad_weights = self.qw.ctypes.data
        r = self.rule
        a.npairs = r.npairs
        a.test_points, a.trial_points, a.weights = ptr(r.test_points), ptr(r.trial_points), ptr(r.weights)
        a.test_elements, a.trial_elements = ptr(r.test_elements), ptr(r.trial_elements)
        a.test_offsets, a.trial_offsets = ptr(r.test_offsets), ptr(r.trial_offsets)
        a.weights_offsets, a.npoints = ptr(r.weights_offsets), ptr(r.npoints)
        a.directions = ptr(self.directions)
        a.ff_dlp_coeff = 1.0
        a.ff_eta[0], a.ff_eta[1] = 0.0, -float(k)
        a.ff_deta_dk[0], a.ff_deta_dk[1] = 0.0, -1.0
        for c in range(3):
            a.incident[c] = self.incident[c]
        a.rhs_coeff[0], a.rhs_coeff[1] = -1.0, 0.0
        a.phase_radius = 1.0001 * 2.0 * geometry.radius
        return a

    def descriptor(self, k):
        return OperatorDescriptor("helmholtz_combined_field_boundary", [float(k), 0.0, 0.0, -float(k)],
                                  "helmholtz_combined_field", "default_scalar", "double", True, None, 1)

    def assemble(self, geometry, k, out=None):
        """A = DLP - 1/2 I - i k SLP (complex128, ne x ne) on the device."""
        n = self.base.nelements
        if out is None:
            out = _torch.empty((n, n), dtype=_torch.complex128, device="cuda")
        desc = self.descriptor(k)
        regular_into(out, desc, self.space, self.space, self.parameters, precision=_lib.FP64, overwrite=True,
                     geometry=geometry)
        singular_into_dense(out, desc, self.space, self.space, self.parameters, diag_shift=-0.5, geometry=geometry)
        return out

    def rhs(self, geometry, k):
        b = _torch.empty(self.base.nelements, dtype=_torch.complex128, device="cuda")
        a = self._args(geometry, k)
        a.out = ptr(b)
        _lib.check(_lib.load().bemppcuda_plane_wave_dp0(_ct.byref(a), current_stream()))
        return b

    def farfield_matrix(self, geometry, k):
        f = _torch.empty((self.directions.shape[0], self.base.nelements), dtype=_torch.complex128, device="cuda")
        a = self._args(geometry, k)
        a.out = ptr(f)
        _lib.check(_lib.load().bemppcuda_farfield_matrix_dp0(_ct.byref(a), current_stream()))
        return f

    # ------------------------------------------------------------------ objective and gradient
    def _gmres(self, matvec, rhs):
        from .linalg import gmres_tensor

        x, info, res, its = gmres_tensor(matvec, rhs, tol=self.tol, restart=300, maxiter=3000, check_every=16,
                                         graph=True)
        if info != 0:
            raise RuntimeError("GMRES did not reach %g in %d iterations (last residual %g)" % (self.tol, its, res[-1]))
        return x, its

    def _gmres32(self, matvec, matvec_low, rhs):
        """Inner GMRES on the complex64 copy, complex128 residuals, to relative residual ``tol``."""
        from .linalg import refine_gmres

        x, info = refine_gmres(matvec, matvec_low, rhs, tol=self.tol, inner_tol=1e-5, restart=300, maxiter=3000,
                               check_every=16)
        if not info["converged"]:
            raise RuntimeError("refined GMRES did not reach %g (residuals %s)" % (self.tol, info["relative_residuals"]))
        return x, sum(info["inner_iterations"])

    def _refine(self, lu, pivots, matvec, rhs, adjoint=False, max_steps=20):
        """Solve with complex64 factors and complex128 residuals; returns (x, steps)."""
        bnorm = float(_torch.linalg.vector_norm(rhs).item())
        x = _torch.zeros_like(rhs)
        r = rhs
        for step in range(1, max_steps + 1):
            d = _torch.linalg.lu_solve(lu, pivots, r.to(_torch.complex64).unsqueeze(1), adjoint=adjoint).squeeze(1)
            x = x + d.to(_torch.complex128)
            r = rhs - matvec(x)
            if float(_torch.linalg.vector_norm(r).item()) <= self.tol * bnorm:
                return x, step
        raise RuntimeError("refinement did not reach %g in %d steps" % (self.tol, max_steps))

    def evaluate(self, vertices, k, keep=False, solver=None):
        """J as a 0-d device tensor (and the state for ``gradient`` when ``keep``)."""
        solver = solver or self.solver
        geometry = self.geometry(vertices)
        a = self.assemble(geometry, k)
        b = self.rhs(geometry, k)
        lu = pivots = matrix = its = None
        if solver == "lu":
            lu, pivots = _torch.linalg.lu_factor(a)
            del a
            phi = _torch.linalg.lu_solve(lu, pivots, b.unsqueeze(1)).squeeze(1)
        elif solver == "lu32":
            matrix = a
            lu, pivots = _torch.linalg.lu_factor(a.to(_torch.complex64))
            phi, its = self._refine(lu, pivots, matvec_of(matrix), b)
        elif solver == "gmres32":
            matrix = a
            low = a.to(_torch.complex64)
            phi, its = self._gmres32(matvec_of(matrix), matvec_of(low), b)
        else:
            matrix = a
            phi, its = self._gmres(matvec_of(matrix), b)
        farfield = self.farfield_matrix(geometry, k)
        u = farfield @ phi
        value = (u.real ** 2 + u.imag ** 2).sum()
        if keep:
            # the complex64 copy (gmres32) serves the adjoint solve too
            return value, ScatteringState(geometry, lu, pivots, phi, u, farfield, matrix, its,
                                          low if solver == "gmres32" else None)
        return value

    def adjoint(self, state):
        """lambda with A^H lambda = F^H u (same solver as the forward solve)."""
        rhs = state.farfield.conj().transpose(0, 1) @ state.u
        if state.lu is not None and state.matrix is not None:  # complex64 factors, refined
            ah = state.matrix.mH
            lam, steps = self._refine(state.lu, state.pivots, lambda v: _torch.mv(ah, v), rhs, adjoint=True)
            return lam
        if state.lu is not None:
            return _torch.linalg.lu_solve(state.lu, state.pivots, rhs.unsqueeze(1), adjoint=True).squeeze(1)
        from .linalg import adjoint_matvec

        if getattr(state, "low", None) is not None:
            lam, its = self._gmres32(adjoint_matvec(state.matrix), adjoint_matvec(state.low), rhs)
            return lam
        lam, its = self._gmres(adjoint_matvec(state.matrix), rhs)
        return lam

    def gradient(self, state, k, lam=None, scales=(-2.0, 2.0, 2.0)):
        """(dJ/dvertices (nv, 3), dJ/dk) from a kept forward state."""
        if lam is None:
            lam = self.adjoint(state)
        vgrad = _torch.zeros((self.base.nvertices, 3), dtype=_torch.float64, device="cuda")
        kgrad = _torch.zeros(1, dtype=_torch.float64, device="cuda")
        a = self._args(state.geometry, k)
        a.phi = ptr(state.phi)
        a.lam = ptr(lam)
        a.u = ptr(state.u)
        a.scale_operator, a.scale_farfield, a.scale_rhs = (float(s) for s in scales)
        a.vertex_grad = ptr(vgrad)
        a.k_grad = ptr(kgrad)
        a.workspace = ptr(self.workspace)
        a.workspace_bytes = self.workspace.numel() * 8
        keep = (lam, state.phi, state.u)
        _lib.check(_lib.load().bemppcuda_shape_adjoint_dp0(_ct.byref(a), current_stream()))
        del keep
        return vgrad, kgrad[0]


class _ObjectiveFunction(_torch.autograd.Function):
    """torch.autograd.Function around FarFieldObjective: forward solve, adjoint backward."""

    @staticmethod
    def forward(ctx, vertices, k, objective):
        kval = float(k.detach().item()) if isinstance(k, _torch.Tensor) else float(k)
        value, state = objective.evaluate(vertices, kval, keep=True)
        ctx.objective = objective
        ctx.state = state
        ctx.kval = kval
        ctx.k_like = k if isinstance(k, _torch.Tensor) else None
        return value

    @staticmethod
    def backward(ctx, grad_output):
        vgrad, kgrad = ctx.objective.gradient(ctx.state, ctx.kval)
        ctx.state = None
        g = grad_output.to(_torch.float64)
        gk = None
        if ctx.k_like is not None:
            gk = (g * kgrad).reshape(ctx.k_like.shape).to(device=ctx.k_like.device, dtype=ctx.k_like.dtype)
        ctx.k_like = None
        return g * vgrad, gk, None


def far_field_objective(vertices, k, objective):
    """J(vertices, k) with autograd support (vertices (nv, 3) float64 CUDA tensor, k a 0-d tensor or float)."""
    return _ObjectiveFunction.apply(vertices, k, objective)
