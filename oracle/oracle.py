"""CPU oracle for the dense assembly / potential path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

The arithmetic lives in ``bempp_oracle.c`` (a plain-C restatement of the
reference Numba kernels); this module reproduces the orchestration of the
reference around those kernels:

* ``assemble_dense``      -> core/dense_assembler.py:49-98 (regular pass per
  test colour as in numba_assemblers.py:58-112, then the singular part
  scattered with ``np.add.at`` and the global multipliers)
* ``singular_values``     -> core/singular_assembler.py:69-142 (flat per-pair
  values plus local row / column indices)
* ``evaluate_potential``  -> core/dense_potential_assembler.py:8-40 and
  numba_assemblers.py:115-164

Inputs are duck-typed "space" objects exposing ``grid.vertices``,
``grid.elements``, ``local2global``, ``local_multipliers``,
``normal_multipliers``, ``support``, ``support_elements``,
``number_of_shape_functions``, ``global_dof_count``, ``localised_space``,
``map_to_full_grid`` and ``get_elements_by_color`` (both the reference's
``FunctionSpace`` and ``bempp_cuda.space.FunctionSpace`` qualify), plus the
singular pair arrays of ``_SingularQuadratureRuleInterfaceGalerkin.get_arrays``.
"""

import ctypes as _ct
import os as _os
import subprocess as _sp

import numpy as _np

_HERE = _os.path.dirname(_os.path.abspath(__file__))
_LIB_PATH = _os.path.join(_HERE, "_build", "libbempp_oracle.so")
_lib = None

KERNELS = {
    "laplace_single_layer": 0,
    "laplace_double_layer": 1,
    "laplace_adjoint_double_layer": 2,
    "helmholtz_single_layer": 3,
    "helmholtz_double_layer": 4,
    "helmholtz_adjoint_double_layer": 5,
    "modified_helmholtz_single_layer": 6,
    "modified_helmholtz_double_layer": 7,
    "modified_helmholtz_adjoint_double_layer": 8,
    "helmholtz_far_field_single_layer": 9,
    "helmholtz_far_field_double_layer": 10,
    "helmholtz_combined_field": 11,
}

ASSEMBLY = {
    "default_scalar": 0,
    "laplace_hypersingular": 1,
    "helmholtz_hypersingular": 2,
    "modified_helmholtz_hypersingular": 3,
    "maxwell_electric_field": 4,
    "maxwell_magnetic_field": 5,
    "maxwell_electric_far_field": 4,
    "maxwell_magnetic_far_field": 5,
}


def build():
    """Compile the C oracle with make (gcc, OpenMP)."""
    _sp.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not _os.path.exists(_LIB_PATH):
            build()
        _lib = _ct.CDLL(_LIB_PATH)
        for name in ("oracle_regular", "oracle_singular", "oracle_potential"):
            getattr(_lib, name).restype = _ct.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(_ct.c_void_p)


def _i64(v):
    return _ct.c_int64(int(v))


def _params(options):
    p = _np.zeros(4, dtype=_np.float64)
    opts = _np.asarray(options, dtype=_np.float64).ravel()
    p[: len(opts)] = opts
    return p


def _grid_arrays(space):
    v = _np.asfortranarray(space.grid.vertices, dtype=_np.float64)
    e = _np.asfortranarray(space.grid.elements, dtype=_np.uint32)
    return v, e


def regular_part(kernel_type, assembly_type, options, domain, dual_to_range, quad_points, quad_weights, result):
    """Accumulate the regular-pair part into ``result`` (rows, cols), colour by colour."""
    lib_ = lib()
    v, e = _grid_arrays(dual_to_range)
    params = _params(options)
    is_complex = int(_np.iscomplexobj(result))
    test_idx, test_ptr = dual_to_range.get_elements_by_color()
    trial = _np.ascontiguousarray(domain.support_elements, dtype=_np.uint32)
    qp = _np.ascontiguousarray(_np.asarray(quad_points, dtype=_np.float64).T)  # (nq, 2)
    qw = _np.ascontiguousarray(quad_weights, dtype=_np.float64)
    args_common = (
        _ct.c_int(ASSEMBLY[assembly_type]),
        _ct.c_int(KERNELS[kernel_type]),
        _p(params),
        _p(v),
        _i64(v.shape[1]),
        _p(e),
        _i64(e.shape[1]),
        _ct.c_int(dual_to_range.number_of_shape_functions),
        _ct.c_int(domain.number_of_shape_functions),
    )
    tm = _np.ascontiguousarray(dual_to_range.local_multipliers, dtype=_np.float64)
    sm = _np.ascontiguousarray(domain.local_multipliers, dtype=_np.float64)
    tl = _np.ascontiguousarray(dual_to_range.local2global, dtype=_np.uint32)
    sl = _np.ascontiguousarray(domain.local2global, dtype=_np.uint32)
    tn = _np.ascontiguousarray(dual_to_range.normal_multipliers, dtype=_np.int32)
    sn = _np.ascontiguousarray(domain.normal_multipliers, dtype=_np.int32)
    grids_identical = int(domain.grid == dual_to_range.grid)
    assert result.flags.c_contiguous
    for c in range(len(test_ptr) - 1):
        tests = _np.ascontiguousarray(test_idx[test_ptr[c] : test_ptr[c + 1]], dtype=_np.uint32)
        lib_.oracle_regular(
            *args_common,
            _p(tests),
            _i64(len(tests)),
            _p(trial),
            _i64(len(trial)),
            _p(tm),
            _p(sm),
            _p(tl),
            _p(sl),
            _p(tn),
            _p(sn),
            _p(qp),
            _p(qw),
            _i64(len(qw)),
            _ct.c_int(grids_identical),
            _p(result),
            _i64(result.shape[1]),
            _ct.c_int(is_complex),
        )


def singular_kernel(kernel_type, assembly_type, options, domain, dual_to_range, rule_arrays, result):
    """Per-pair singular values (numba_assemblers.py:6-55) accumulated into flat ``result``."""
    (tp, sp, w, te, se, toff, soff, woff, npts) = rule_arrays
    v, e = _grid_arrays(domain)
    params = _params(options)
    tp = _np.ascontiguousarray(_np.asarray(tp, dtype=_np.float64).T)
    sp = _np.ascontiguousarray(_np.asarray(sp, dtype=_np.float64).T)
    arrs = [_np.ascontiguousarray(a, dtype=_np.uint32) for a in (te, se, toff, soff, woff, npts)]
    w = _np.ascontiguousarray(w, dtype=_np.float64)
    lib().oracle_singular(
        _ct.c_int(ASSEMBLY[assembly_type]),
        _ct.c_int(KERNELS[kernel_type]),
        _p(params),
        _p(v),
        _i64(v.shape[1]),
        _p(e),
        _i64(e.shape[1]),
        _ct.c_int(dual_to_range.number_of_shape_functions),
        _ct.c_int(domain.number_of_shape_functions),
        _p(tp),
        _p(sp),
        _p(w),
        *[_p(a) for a in arrs],
        _i64(len(arrs[0])),
        _p(_np.ascontiguousarray(dual_to_range.normal_multipliers, dtype=_np.int32)),
        _p(_np.ascontiguousarray(domain.normal_multipliers, dtype=_np.int32)),
        _p(result),
        _ct.c_int(int(_np.iscomplexobj(result))),
    )


def singular_values(kernel_type, assembly_type, options, domain, dual_to_range, rule_arrays, is_complex):
    """Return (local rows, local cols, values) of the singular part (singular_assembler.py:69-142)."""
    nt = dual_to_range.number_of_shape_functions
    ns = domain.number_of_shape_functions
    te, se = rule_arrays[3], rule_arrays[4]
    npairs = len(te)
    result = _np.zeros(nt * ns * npairs, dtype=_np.complex128 if is_complex else _np.float64)
    singular_kernel(kernel_type, assembly_type, options, domain, dual_to_range, rule_arrays, result)
    irange = _np.arange(nt)
    jrange = _np.arange(ns)
    i_ind = _np.tile(_np.repeat(irange, ns), npairs) + _np.repeat(te.astype(_np.int64) * nt, nt * ns)
    j_ind = _np.tile(_np.tile(jrange, nt), npairs) + _np.repeat(se.astype(_np.int64) * ns, nt * ns)
    return i_ind, j_ind, result


def assemble_dense(
    kernel_type,
    assembly_type,
    options,
    is_complex,
    domain,
    dual_to_range,
    quad_points,
    quad_weights,
    rule_arrays=None,
):
    """Dense weak form: regular pass plus singular correction (dense_assembler.py:49-98).

    ``rule_arrays`` are the singular pair arrays built on the localised spaces
    (required when the two spaces share a grid).
    """
    rows = dual_to_range.global_dof_count
    cols = domain.global_dof_count
    result = _np.zeros((rows, cols), dtype=_np.complex128 if is_complex else _np.float64)
    regular_part(kernel_type, assembly_type, options, domain, dual_to_range, quad_points, quad_weights, result)
    if domain.grid == dual_to_range.grid:
        if rule_arrays is None:
            raise ValueError("singular rule arrays are required for identical grids")
        i_loc, j_loc, vals = singular_values(
            kernel_type,
            assembly_type,
            options,
            domain.localised_space,
            dual_to_range.localised_space,
            rule_arrays,
            is_complex,
        )
        t_l2g = dual_to_range.local2global.ravel()
        s_l2g = domain.local2global.ravel()
        t_mul = dual_to_range.local_multipliers.ravel()
        s_mul = domain.local_multipliers.ravel()
        # i_loc / j_loc are element * nshape + local index slots (singular_assembler.py:132-142)
        rr = i_loc
        cc = j_loc
        _np.add.at(result, (t_l2g[rr], s_l2g[cc]), vals * s_mul[cc] * t_mul[rr])
    return result


class _RowSample(object):
    """The dual space seen through a row sample: only the test elements that touch a sampled dof
    are in the support, and ``local2global`` sends every dof to its position in the sample, or to
    one discard row (index ``len(rows)``) for dofs outside it.  A sampled row then receives every
    contribution the full assembly gives it, regular and singular, since all its test elements
    are kept."""

    def __init__(self, space, rows):
        rows = _np.asarray(rows, dtype=_np.int64)
        nshape = space.number_of_shape_functions
        rowmap = _np.full(space.global_dof_count, len(rows), dtype=_np.int64)
        rowmap[rows] = _np.arange(len(rows))
        l2g = _np.asarray(space.local2global, dtype=_np.int64).reshape(-1, nshape)
        support = _np.asarray(space.support, dtype=bool)
        touch = support & _np.isin(l2g, rows).any(axis=1)
        self.grid = space.grid
        self.support = touch
        self.support_elements = _np.flatnonzero(touch).astype(_np.uint32)
        self.local2global = _np.where(support[:, None], rowmap[_np.where(support[:, None], l2g, 0)],
                                      len(rows)).astype(_np.uint32)
        self.local_multipliers = space.local_multipliers
        self.normal_multipliers = space.normal_multipliers
        self.number_of_shape_functions = nshape
        self.global_dof_count = len(rows) + 1
        self.localised_space = space.localised_space
        idx, ptr = space.get_elements_by_color()
        idx = _np.asarray(idx)
        keep = touch[idx]
        counts = _np.add.reduceat(keep.astype(_np.int64), _np.asarray(ptr[:-1])) if len(idx) else []
        self._colors = (idx[keep], _np.concatenate([[0], _np.cumsum(counts)]).astype(_np.int64))

    def get_elements_by_color(self):
        return self._colors


def assemble_rows(kernel_type, assembly_type, options, is_complex, domain, dual_to_range, rows, quad_points,
                  quad_weights, singular_order=4):
    """Rows ``rows`` (global dofs of ``dual_to_range``) of the dense weak form, regular plus singular part.

    Equal to ``assemble_dense(...)[rows]`` (dense_assembler.py:49-98) at the cost of the sampled rows only:
    a parity check of a matrix too large for the oracle to assemble whole.
    """
    from bempp_cuda.quadrature import SingularPairs

    view = _RowSample(dual_to_range, rows)
    rule = None
    if domain.grid == dual_to_range.grid:
        rule = SingularPairs(domain.grid, singular_order, view.support, domain.support).arrays()
    full = assemble_dense(kernel_type, assembly_type, options, is_complex, domain, view, quad_points, quad_weights,
                          rule)
    return full[: len(rows)]


def evaluate_potential(kernel_type, assembly_type, options, space, points, coefficients, quad_points, quad_weights):
    """Potential values (kdim, npoints) for global coefficients ``coefficients``."""
    kdim = 3 if assembly_type.startswith("maxwell") else 1
    local = space.map_to_full_grid @ _np.asarray(coefficients)
    x = _np.ascontiguousarray(local, dtype=_np.complex128)
    v, e = _grid_arrays(space)
    pts = _np.ascontiguousarray(_np.asarray(points, dtype=_np.float64).T)
    qp = _np.ascontiguousarray(_np.asarray(quad_points, dtype=_np.float64).T)
    qw = _np.ascontiguousarray(quad_weights, dtype=_np.float64)
    sup = _np.ascontiguousarray(space.support_elements, dtype=_np.uint32)
    result = _np.zeros((kdim, pts.shape[0]), dtype=_np.complex128)
    lib().oracle_potential(
        _ct.c_int(ASSEMBLY[assembly_type]),
        _ct.c_int(KERNELS[kernel_type]),
        _p(_params(options)),
        _p(v),
        _i64(v.shape[1]),
        _p(e),
        _i64(e.shape[1]),
        _ct.c_int(space.number_of_shape_functions),
        _p(sup),
        _i64(len(sup)),
        _p(_np.ascontiguousarray(space.normal_multipliers, dtype=_np.int32)),
        _p(qp),
        _p(qw),
        _i64(len(qw)),
        _p(pts),
        _i64(pts.shape[0]),
        _p(x),
        _p(result),
    )
    return result
