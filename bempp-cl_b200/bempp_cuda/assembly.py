"""Dense assembly and potential evaluation on the device.

``assemble_dense_device`` is the fused replacement of
``bempp_cl.core.dense_assembler.assemble_dense`` (core/dense_assembler.py:49-98):
the regular pass and the singular correction both run on the GPU and the
matrix stays in HBM as a torch tensor.  The functions below take the
reference's own descriptor / space / parameter objects (duck-typed: a
``bempp_cl`` object and the matching ``bempp_cuda`` object both work).

Precision: ``device_interface`` "cuda" is FP64 end to end; "cuda_mixed"
evaluates the regular pairs in FP32 where the library has a mixed kernel
(DP0 scalar kernels; P1 single, double, adjoint double layer and
hypersingular operators, P1 beside P0; the Maxwell electric and magnetic
fields; scalar potentials, Helmholtz far fields and the Maxwell magnetic
potential and far field) and keeps the singular pairs, per-entry sums and
element-pair factors in FP64.  Operators without a mixed kernel run in FP64
and say so once (``MixedPrecisionFallback``).
"""

import numpy as _np
import torch as _torch

from . import _lib
from .device import (
    current_stream,
    device_grid,
    device_singular_rule,
    device_space,
    ptr,
    require_cuda,
)
from .quadrature import number_of_duffy_points, triangle_rule

_REG_CACHE = {}


def precision_of(device_interface):
    parts = str(device_interface).split("_")
    if parts[0] != "cuda":
        raise ValueError("device interface %r is not a cuda interface" % (device_interface,))
    if len(parts) > 1 and parts[1] == "mixed":
        return _lib.MIXED
    return _lib.FP64


def kernel_ids(descriptor):
    try:
        kernel = _lib.KERNEL_IDS[descriptor.kernel_type]
        assembly = _lib.ASSEMBLY_IDS[descriptor.assembly_type]
    except KeyError as exc:
        raise ValueError("operator %r is not supported by the cuda interface" % (descriptor.identifier,)) from exc
    return kernel, assembly


def kernel_params(options):
    p = _np.zeros(4, dtype=_np.float64)
    opts = _np.asarray(options, dtype=_np.float64).ravel()
    if len(opts) > 4:
        raise ValueError("at most four kernel options are supported")
    p[: len(opts)] = opts
    return p


def _set_params(args, options):
    p = kernel_params(options)
    for i in range(4):
        args.params[i] = float(p[i])


def regular_rule(order):
    key = int(order)
    if key not in _REG_CACHE:
        points, weights = triangle_rule(key)
        _REG_CACHE[key] = (_np.ascontiguousarray(points.T), _np.ascontiguousarray(weights))
    return _REG_CACHE[key]


def _grids_identical(domain, dual_to_range):
    return domain.grid == dual_to_range.grid


def same_space(a, b):
    """True when two spaces are the same discretisation of one grid (so one device copy serves both)."""
    if a is b:
        return True
    try:
        if a.grid is not b.grid or a.shapeset.identifier != b.shapeset.identifier:
            return False
        if int(a.global_dof_count) != int(b.global_dof_count):
            return False
        return all(_np.array_equal(_np.asarray(getattr(a, f)), _np.asarray(getattr(b, f)))
                   for f in ("support_elements", "local2global", "local_multipliers", "normal_multipliers"))
    except AttributeError:
        return False


def regular_into(
    result, descriptor, domain, dual_to_range, parameters, precision=_lib.FP64, overwrite=False, stream=None,
    geometry=None, symmetric=True, rows=None, result_is_zero=False, tresult=None, col_begin=0,
):
    """Add (or with ``overwrite`` store) the regular part into the device tensor ``result``.

    ``geometry`` (a DeviceGrid-like object with ``record()`` and ``radius``)
    replaces the device geometry of both grids, e.g. a grid whose vertices
    moved while its elements stayed the same.  With ``symmetric`` (default)
    the library computes A_ij and A_ji from one sweep when both spaces are the
    same DP0 space of one grid; ``symmetric=False`` evaluates every entry on
    its own.  ``rows=(lo, hi)`` restricts a symmetric sweep to the pairs
    (i, j), i <= j, with rows i in [lo, hi) (both entries written).
    ``result_is_zero`` promises that ``result`` holds zeros, which lets
    symmetric P1 single-layer and hypersingular sweeps add only the blocks
    of the pairs i < j and symmetrise the matrix afterwards.  ``tresult``
    (with ``rows``, DP0 symmetric sweep): stripe mode, ``result`` and
    ``tresult`` hold rows [lo, hi) and columns [col_begin, n): A_ij of the
    swept pairs i <= j at result[i - lo, j - col_begin], A_ji at
    tresult[i - lo, j - col_begin].
    """
    require_cuda()
    kernel, assembly = kernel_ids(descriptor)
    if result.numel() == 0:
        return result  # a space without dofs: nothing to assemble
    tgrid = geometry or device_grid(dual_to_range.grid)
    sgrid = geometry or device_grid(domain.grid)
    sspace = device_space(domain)
    # an equal dual space shares the domain's device copy, which lets the
    # library take the symmetric sweep (it compares the pointers)
    tspace = sspace if same_space(domain, dual_to_range) else device_space(dual_to_range)
    points, weights = regular_rule(parameters.quadrature.regular)
    args = _lib.RegularArgs()
    args.kernel = kernel
    args.assembly = assembly
    args.precision = precision
    args.is_complex = 1 if result.is_complex() else 0
    _set_params(args, descriptor.options)
    args.test_grid = tgrid.record()
    args.trial_grid = sgrid.record()
    args.test = tspace.record()
    args.trial = sspace.record()
    args.grids_identical = 1 if _grids_identical(domain, dual_to_range) else 0
    args.nq = len(weights)
    args.quad_points = points.ctypes.data
    args.quad_weights = weights.ctypes.data
    args.result = ptr(result)
    args.ld = result.stride(0)
    args.overwrite = 1 if overwrite else 0
    args.no_symmetry = 0 if symmetric else 1
    args.result_is_zero = 1 if result_is_zero else 0
    if rows is not None:
        args.row_begin, args.row_end = int(rows[0]), int(rows[1])
    if tresult is not None:
        if tresult.shape != result.shape or tresult.dtype != result.dtype or tresult.stride() != result.stride():
            raise ValueError("tresult must have the shape, dtype and strides of result")
        args.tresult = ptr(tresult)
        args.col_begin = int(col_begin)
    # a little slack over the exact bound keeps rounding of the radii on the safe side
    args.phase_radius = 1.0001 * (tgrid.radius + sgrid.radius)
    _lib.check(_lib.load().bemppcuda_assemble_regular(args, stream or current_stream()))
    return result


def apply_regular(y, x, descriptor, domain, dual_to_range, parameters, stream=None):
    """y += A_reg x in FP64, A_reg the regular part evaluated on the fly (bemppcuda_apply_regular).

    One DP0 space of one grid on both sides (Laplace / Helmholtz single, double,
    adjoint double layer, combined field); ``x``, ``y`` complex128 device
    vectors.  The adjacent pairs (the singular part) contribute nothing.
    """
    require_cuda()
    if not same_space(domain, dual_to_range):
        raise ValueError("apply_regular needs the same DP0 space on both sides")
    kernel, assembly = kernel_ids(descriptor)
    space = device_space(domain)
    grid = device_grid(domain.grid)
    points, weights = regular_rule(parameters.quadrature.regular)
    args = _lib.RegularArgs()
    args.kernel = kernel
    args.assembly = assembly
    args.precision = _lib.FP64
    args.is_complex = 1
    _set_params(args, descriptor.options)
    args.test_grid = args.trial_grid = grid.record()
    args.test = args.trial = space.record()
    args.grids_identical = 1
    args.nq = len(weights)
    args.quad_points = points.ctypes.data
    args.quad_weights = weights.ctypes.data
    args.phase_radius = 1.0001 * 2.0 * grid.radius
    _lib.check(_lib.load().bemppcuda_apply_regular(args, ptr(x), ptr(y), stream or current_stream()))
    return y


def adjacent_part(matrix, domain, dual_to_range, parameters):
    """The entries of a dense DP0 weak form at the adjacent element pairs (the singular part, with any
    identity term), as a device CSR matrix.  Both spaces map element e to dof e (same DP0 space)."""
    grid = domain.grid
    n = grid.number_of_elements
    if not (same_space(domain, dual_to_range) and device_space(domain).dof_is_position
            and int(domain.global_dof_count) == n and tuple(matrix.shape) == (n, n)):
        raise ValueError("adjacent_part needs one DP0 space on every element of the grid on both sides")
    rule = device_singular_rule(grid, parameters.quadrature.singular, dual_to_range.support, domain.support)
    te, se = (_torch.as_tensor(a.astype(_np.int64), device=matrix.device) for a in rule._host_ints[:2])
    keys = _torch.unique(te * matrix.shape[1] + se)
    rows, cols = keys // matrix.shape[1], keys % matrix.shape[1]
    vals = matrix[rows, cols]
    crow = _torch.zeros(matrix.shape[0] + 1, dtype=_torch.int64, device=matrix.device)
    crow[1:] = _torch.cumsum(_torch.bincount(rows, minlength=matrix.shape[0]), 0)
    return _torch.sparse_csr_tensor(crow, cols, vals, size=tuple(matrix.shape))


def basis_kind(space):
    """BEMPPCUDA_BASIS_* of a space: RWG, SNC (n x RWG) or scalar."""
    ident = getattr(space, "identifier", "")
    if ident.startswith("rwg"):
        return _lib.BASIS_RWG
    if ident.startswith("snc"):
        return _lib.BASIS_SNC
    return _lib.BASIS_SCALAR


def identity_triplets(domain, dual_to_range, parameters, stream=None):
    """COO triplets (rows, cols, values) of the L2 identity on the device (csrc/identity.cu).

    The reference (core/sparse_assembler.py:17-70) evaluates the same local
    mass matrices on the elements of both supports and sums repeated (row,
    col) pairs when it converts to CSR; the caller does that here.
    """
    require_cuda()
    if domain.grid != dual_to_range.grid:
        raise ValueError("For sparse operators the domain and dual_to_range grids must be identical.")
    tk, sk = basis_kind(dual_to_range), basis_kind(domain)
    if (tk == _lib.BASIS_SCALAR) != (sk == _lib.BASIS_SCALAR):
        raise ValueError("the identity needs two scalar spaces or two RWG / SNC spaces")
    elements = _np.flatnonzero(_np.asarray(domain.support) & _np.asarray(dual_to_range.support)).astype(_np.int32)
    nt = int(dual_to_range.number_of_shape_functions)
    ns = int(domain.number_of_shape_functions)
    n = len(elements) * nt * ns
    rows = _torch.empty(n, dtype=_torch.int64, device="cuda")
    cols = _torch.empty(n, dtype=_torch.int64, device="cuda")
    values = _torch.empty(n, dtype=_torch.float64, device="cuda")
    if n == 0:
        return rows, cols, values
    el = _torch.as_tensor(elements).to("cuda")
    grid = device_grid(domain.grid)
    sspace = device_space(domain)
    tspace = sspace if same_space(domain, dual_to_range) else device_space(dual_to_range)
    points, weights = regular_rule(parameters.quadrature.regular)
    args = _lib.IdentityArgs()
    args.grid = grid.record()
    args.test = tspace.record()
    args.trial = sspace.record()
    args.test_kind, args.trial_kind = tk, sk
    args.nelements = len(elements)
    args.elements = ptr(el)
    args.nq = len(weights)
    args.quad_points = points.ctypes.data
    args.quad_weights = weights.ctypes.data
    args.rows, args.cols, args.values = ptr(rows), ptr(cols), ptr(values)
    _lib.check(_lib.load().bemppcuda_assemble_identity(args, stream or current_stream()))
    return rows, cols, values


def dp0_fast_path(descriptor, domain, dual_to_range, parameters):
    """True when the regular pass can overwrite every entry (no pre-zeroing needed)."""
    if descriptor.assembly_type != "default_scalar":
        return False
    if int(parameters.quadrature.regular) != 4:
        return False
    return bool(device_space(domain).dof_is_position and device_space(dual_to_range).dof_is_position)


def singular_into_dense(result, descriptor, domain, dual_to_range, parameters, diag_shift=0.0, stream=None,
                        geometry=None, rows=None, mirror=True):
    """Scatter the Sauter-Schwab pairs into the dense device tensor ``result`` (``geometry`` as in regular_into).

    ``rows=(lo, hi)``: only the pairs whose test element is one of the support
    elements lo .. hi-1 of ``dual_to_range`` (support in increasing order).
    ``mirror`` (default) lets the DP0 kernel evaluate each vertex-adjacent pair
    once for both orders when both spaces are the same; ``mirror=False``
    evaluates every ordered pair on its own.
    """
    kernel, assembly = kernel_ids(descriptor)
    if result.numel() == 0:
        return result
    grid = domain.grid
    rule = device_singular_rule(grid, parameters.quadrature.singular, dual_to_range.support, domain.support)
    args = _lib.SingularArgs()
    args.kernel = kernel
    args.assembly = assembly
    args.is_complex = 1 if result.is_complex() else 0
    _set_params(args, descriptor.options)
    args.grid = (geometry or device_grid(grid)).record()
    args.test = device_space(dual_to_range).record()
    args.trial = device_space(domain).record()
    if rows is None:
        rule.fill(args)
    else:
        sup = _np.asarray(dual_to_range.support_elements)
        rule.fill(args, rule.pair_range(int(sup[rows[0]]), int(sup[rows[1] - 1])))
    args.values = None
    args.dense = ptr(result)
    args.ld = result.stride(0)
    args.diag_shift = float(diag_shift)
    args.phase_radius = 1.0001 * 2.0 * (geometry or device_grid(grid)).radius
    if mirror and same_space(domain, dual_to_range):
        # every pair is listed in both orders and the vertex-adjacent rule (its weights follow the
        # coincident and edge-adjacent ones) is symmetric in test and trial points: the DP0 kernel
        # evaluates each such pair once for both entries
        order = parameters.quadrature.singular
        args.mirror_weights_offset = (number_of_duffy_points(order, "coincident")
                                      + number_of_duffy_points(order, "edge_adjacent"))
    _lib.check(_lib.load().bemppcuda_assemble_singular(args, stream or current_stream()))
    return result


class MixedPrecisionFallback(UserWarning):
    """device_interface="cuda_mixed" asked for an operator that has no mixed-precision kernel: it is
    assembled / evaluated in FP64 (same values as "cuda")."""


FP64_FALLBACKS = set()


def note_fp64_fallback(descriptor, what):
    """Record (and warn once per operator kind) that a mixed-precision request ran in FP64."""
    import warnings

    key = (what, getattr(descriptor, "kernel_type", None), getattr(descriptor, "assembly_type", None))
    if key not in FP64_FALLBACKS:
        FP64_FALLBACKS.add(key)
        warnings.warn("cuda_mixed: no mixed-precision %s kernel for %s / %s; evaluated in FP64"
                      % (what, key[1], key[2]), MixedPrecisionFallback, stacklevel=3)


def _regular_with_fallback(result, descriptor, domain, dual_to_range, parameters, precision, **kw):
    """``regular_into`` in ``precision``; where the library has no mixed-precision
    kernel for the operator (it says so before launching anything) the FP64 one."""
    try:
        regular_into(result, descriptor, domain, dual_to_range, parameters, precision=precision, **kw)
    except _lib.BemppCudaError as exc:
        if exc.status != _lib.ERR_UNSUPPORTED or precision != _lib.MIXED:
            raise
        note_fp64_fallback(descriptor, "regular-pair")
        regular_into(result, descriptor, domain, dual_to_range, parameters, precision=_lib.FP64, **kw)


def result_dtype(descriptor):
    return _torch.complex128 if descriptor.is_complex else _torch.float64


def assemble_dense_device(domain, dual_to_range, parameters, descriptor, device_interface="cuda", out=None):
    """Full dense weak form (regular + singular) as a device tensor (rows, cols)."""
    require_cuda()
    precision = precision_of(device_interface)
    if getattr(domain, "requires_dof_transformation", False) or getattr(
        dual_to_range, "requires_dof_transformation", False
    ):
        raise ValueError("Spaces that require dof transformations not supported for dense assembly.")
    rows = int(dual_to_range.global_dof_count)
    cols = int(domain.global_dof_count)
    dtype = result_dtype(descriptor)
    fast = dp0_fast_path(descriptor, domain, dual_to_range, parameters)
    if out is None:
        out = _torch.empty((rows, cols), dtype=dtype, device="cuda") if fast else _torch.zeros(
            (rows, cols), dtype=dtype, device="cuda"
        )
    elif not fast:
        out.zero_()
    _regular_with_fallback(out, descriptor, domain, dual_to_range, parameters, precision, overwrite=fast,
                           result_is_zero=not fast)
    if _grids_identical(domain, dual_to_range):
        singular_into_dense(out, descriptor, domain, dual_to_range, parameters)
    return out


def symmetric_rows_eligible(descriptor, domain, dual_to_range, parameters):
    """True when the library can run the symmetric sweep in row blocks (same DP0 space, real k)."""
    if not (dp0_fast_path(descriptor, domain, dual_to_range, parameters) and same_space(domain, dual_to_range)):
        return False
    if descriptor.kernel_type not in ("laplace_single_layer", "laplace_double_layer", "laplace_adjoint_double_layer",
                                      "helmholtz_single_layer", "helmholtz_double_layer",
                                      "helmholtz_adjoint_double_layer", "helmholtz_combined_field"):
        return False
    p = kernel_params(descriptor.options)
    return descriptor.kernel_type.startswith("laplace") or (p[1] == 0.0 and p[0] > 0.0)


def assemble_dense_to_host(domain, dual_to_range, parameters, descriptor, device_interface="cuda", out=None,
                           diag_shift=0.0, blocks=16):
    """Dense DP0 weak form streamed into (pinned) host memory while it is assembled.

    The symmetric sweep runs one row block at a time in row order: after the
    block's upper-triangle tiles (which also write the transposes into later
    rows) and its singular pairs, its rows are final, so their copy to the
    host overlaps the next block's assembly on a second stream.  Other
    operators are assembled whole and then copied.  Returns the host tensor.
    """
    require_cuda()
    rows = int(dual_to_range.global_dof_count)
    cols = int(domain.global_dof_count)
    dtype = result_dtype(descriptor)
    if out is None:
        out = _torch.empty((rows, cols), dtype=dtype, pin_memory=True)
    if not symmetric_rows_eligible(descriptor, domain, dual_to_range, parameters):
        # whole operator on the device, then one copy (the fused-path steps of
        # assemble_combined_field_device, with the identity shift)
        fast = dp0_fast_path(descriptor, domain, dual_to_range, parameters)
        dev = (_torch.empty if fast else _torch.zeros)((rows, cols), dtype=dtype, device="cuda")
        _regular_with_fallback(dev, descriptor, domain, dual_to_range, parameters, precision_of(device_interface),
                               overwrite=fast, result_is_zero=not fast)
        if _grids_identical(domain, dual_to_range):
            singular_into_dense(dev, descriptor, domain, dual_to_range, parameters, diag_shift=diag_shift)
        elif diag_shift != 0.0:
            raise ValueError("an identity term needs identical domain and dual grids")
        out.copy_(dev, non_blocking=True)
        _torch.cuda.current_stream().synchronize()
        return out
    precision = precision_of(device_interface)
    dev = _torch.empty((rows, cols), dtype=dtype, device="cuda")
    compute = _torch.cuda.current_stream()
    copy = _torch.cuda.Stream()
    bounds = [(rows * b) // blocks for b in range(blocks + 1)]
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        if hi <= lo:
            continue
        regular_into(dev, descriptor, domain, dual_to_range, parameters, precision=precision, overwrite=True,
                     rows=(lo, hi))
        singular_into_dense(dev, descriptor, domain, dual_to_range, parameters, diag_shift=diag_shift, rows=(lo, hi))
        done = _torch.cuda.Event()
        done.record(compute)
        copy.wait_event(done)
        with _torch.cuda.stream(copy):
            out[lo:hi].copy_(dev[lo:hi], non_blocking=True)
    compute.wait_stream(copy)
    copy.synchronize()
    del dev
    return out


def assemble_combined_field_device(domain, dual_to_range, parameters, options, eta, identity_coefficient=0.0,
                                   device_interface="cuda", out=None):
    """DP0 Helmholtz DLP + eta * SLP + identity_coefficient * I in one fused pass.

    ``options`` are the Helmholtz kernel options [Re k, Im k].  The identity
    term is the DP0 mass matrix (element areas on the diagonal).
    """
    from .operators import OperatorDescriptor

    opts = list(kernel_params(options)[:2]) + [complex(eta).real, complex(eta).imag]
    desc = OperatorDescriptor("helmholtz_combined_field_boundary", opts, "helmholtz_combined_field", "default_scalar",
                              "double", True, None, 1)
    require_cuda()
    precision = precision_of(device_interface)
    rows = int(dual_to_range.global_dof_count)
    cols = int(domain.global_dof_count)
    fast = dp0_fast_path(desc, domain, dual_to_range, parameters)
    if out is None:
        out = (_torch.empty if fast else _torch.zeros)((rows, cols), dtype=_torch.complex128, device="cuda")
    elif not fast:
        out.zero_()
    regular_into(out, desc, domain, dual_to_range, parameters, precision=precision if fast else _lib.FP64,
                 overwrite=fast)
    if _grids_identical(domain, dual_to_range):
        singular_into_dense(out, desc, domain, dual_to_range, parameters, diag_shift=identity_coefficient)
    elif identity_coefficient != 0.0:
        raise ValueError("an identity term needs identical domain and dual grids")
    return out


def potential_workspace_bytes(args):
    return int(_lib.load().bemppcuda_potential_workspace_bytes(args))


def evaluate_potential_device(space, descriptor, points, local_coefficients, parameters, stream=None,
                              precision=_lib.FP64):
    """Potential (kdim, npoints) complex128 device tensor.

    ``local_coefficients`` are the element-local coefficients (nshape * ne,)
    complex128, i.e. ``space.map_to_full_grid @ x`` of the reference
    (dense_potential_assembler.py:30-34); ``points`` is a (3, npoints) array.
    ``precision=MIXED`` evaluates the point-source pairs of Laplace,
    Helmholtz (real or complex k) and modified Helmholtz single / double
    layer potentials, Helmholtz far fields and the Maxwell magnetic potential
    and far field in FP32; the library refuses it for the Maxwell electric
    potential and far field, which the operator layer then runs in FP64.
    """
    require_cuda()
    kernel, assembly = kernel_ids(descriptor)
    kdim = 3 if assembly in (_lib.ASM_EFIE, _lib.ASM_MFIE) else 1
    dgrid = device_grid(space.grid)
    dspace = device_space(space)
    pts = points if isinstance(points, _torch.Tensor) else _torch.as_tensor(_np.ascontiguousarray(_np.asarray(points, dtype=_np.float64).T))
    pts = pts.to(device="cuda", dtype=_torch.float64).contiguous()
    coeff = local_coefficients
    if not isinstance(coeff, _torch.Tensor):
        coeff = _torch.as_tensor(_np.ascontiguousarray(_np.asarray(coeff, dtype=_np.complex128)))
    coeff = coeff.to(device="cuda", dtype=_torch.complex128).contiguous()
    qp, qw = regular_rule(parameters.quadrature.regular)
    npoints = pts.shape[0]
    result = _torch.empty((kdim, npoints), dtype=_torch.complex128, device="cuda")
    args = _lib.PotentialArgs()
    args.kernel = kernel
    args.assembly = assembly
    _set_params(args, descriptor.options)
    args.grid = dgrid.record()
    args.space = dspace.record()
    args.nq = len(qw)
    args.quad_points = qp.ctypes.data
    args.quad_weights = qw.ctypes.data
    args.npoints = npoints
    args.points = ptr(pts)
    args.coefficients = ptr(coeff)
    args.result = ptr(result)
    need = potential_workspace_bytes(args)
    workspace = _torch.empty(max(need // 8, 1), dtype=_torch.float64, device="cuda")
    args.workspace = ptr(workspace)
    args.workspace_bytes = need
    args.phase_radius = 1.0001 * dgrid.radius
    args.precision = precision
    lib = _lib.load()
    rc = lib.bemppcuda_evaluate_potential(args, stream or current_stream())
    if rc == _lib.ERR_UNSUPPORTED and precision == _lib.MIXED:
        note_fp64_fallback(descriptor, "potential")
        args.precision = _lib.FP64  # no mixed kernel for this potential
        rc = lib.bemppcuda_evaluate_potential(args, stream or current_stream())
    _lib.check(rc)
    return result
