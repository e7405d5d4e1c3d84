"""ctypes binding of libbemppcuda.so (declarations in include/bemppcuda.h).

The library is built in-tree by ``bempp_cuda.build.build()``.  Loading fails
loudly when it is missing: there is no CPU fallback anywhere in this package.
"""

import ctypes as _ct
import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "libbemppcuda.so")

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_UNSUPPORTED = -3
ERR_WORKSPACE = -4

LAPLACE_SLP, LAPLACE_DLP, LAPLACE_ADLP = 0, 1, 2
HELMHOLTZ_SLP, HELMHOLTZ_DLP, HELMHOLTZ_ADLP = 3, 4, 5
MODHELM_SLP, MODHELM_DLP, MODHELM_ADLP = 6, 7, 8
FARFIELD_SLP, FARFIELD_DLP = 9, 10
HELMHOLTZ_COMBINED = 11

ASM_SCALAR, ASM_LAPLACE_HYP, ASM_HELM_HYP, ASM_MODHELM_HYP, ASM_EFIE, ASM_MFIE = range(6)
SHAPE_P0, SHAPE_P1, SHAPE_RWG = 0, 1, 2
FP64, MIXED = 0, 1
GEOM_FIELDS = 25
MAX_REGULAR_POINTS = 16

KERNEL_IDS = {
    "laplace_single_layer": LAPLACE_SLP,
    "laplace_double_layer": LAPLACE_DLP,
    "laplace_adjoint_double_layer": LAPLACE_ADLP,
    "helmholtz_single_layer": HELMHOLTZ_SLP,
    "helmholtz_double_layer": HELMHOLTZ_DLP,
    "helmholtz_adjoint_double_layer": HELMHOLTZ_ADLP,
    "modified_helmholtz_single_layer": MODHELM_SLP,
    "modified_helmholtz_double_layer": MODHELM_DLP,
    "modified_helmholtz_adjoint_double_layer": MODHELM_ADLP,
    "helmholtz_far_field_single_layer": FARFIELD_SLP,
    "helmholtz_far_field_double_layer": FARFIELD_DLP,
    "helmholtz_combined_field": HELMHOLTZ_COMBINED,
}

ASSEMBLY_IDS = {
    "default_scalar": ASM_SCALAR,
    "laplace_hypersingular": ASM_LAPLACE_HYP,
    "helmholtz_hypersingular": ASM_HELM_HYP,
    "modified_helmholtz_hypersingular": ASM_MODHELM_HYP,
    "maxwell_electric_field": ASM_EFIE,
    "maxwell_magnetic_field": ASM_MFIE,
    "maxwell_electric_far_field": ASM_EFIE,
    "maxwell_magnetic_far_field": ASM_MFIE,
}

SHAPESET_IDS = {"p0_discontinuous": SHAPE_P0, "p1_discontinuous": SHAPE_P1, "rwg0": SHAPE_RWG, "snc0": SHAPE_RWG}

_vp = _ct.c_void_p
_i32 = _ct.c_int32
_i64 = _ct.c_int64


class Space(_ct.Structure):
    _fields_ = [
        ("shapeset", _i32),
        ("nshape", _i32),
        ("nsupport", _i64),
        ("support", _vp),
        ("l2g", _vp),
        ("mult", _vp),
        ("normal_mult", _vp),
        ("ndofs", _i64),
        ("dof_is_position", _i32),
        ("pad", _i32),
    ]


class GridRec(_ct.Structure):
    _fields_ = [("nvertices", _i64), ("nelements", _i64), ("geom", _vp), ("elements", _vp)]


class RegularArgs(_ct.Structure):
    _fields_ = [
        ("kernel", _i32),
        ("assembly", _i32),
        ("precision", _i32),
        ("is_complex", _i32),
        ("params", _ct.c_double * 4),
        ("test_grid", GridRec),
        ("trial_grid", GridRec),
        ("test", Space),
        ("trial", Space),
        ("grids_identical", _i32),
        ("nq", _i32),
        ("quad_points", _vp),
        ("quad_weights", _vp),
        ("result", _vp),
        ("ld", _i64),
        ("overwrite", _i32),
        ("no_symmetry", _i32),
        ("phase_radius", _ct.c_double),
        ("row_begin", _i64),
        ("row_end", _i64),
        ("result_is_zero", _i32),
        ("pad2", _i32),
        ("tresult", _vp),
        ("col_begin", _i64),
    ]


class SingularArgs(_ct.Structure):
    _fields_ = [
        ("kernel", _i32),
        ("assembly", _i32),
        ("is_complex", _i32),
        ("pad0", _i32),
        ("params", _ct.c_double * 4),
        ("grid", GridRec),
        ("test", Space),
        ("trial", Space),
        ("npairs", _i64),
        ("npoints_table", _i64),
        ("test_points", _vp),
        ("trial_points", _vp),
        ("weights", _vp),
        ("nweights", _i64),
        ("test_elements", _vp),
        ("trial_elements", _vp),
        ("test_offsets", _vp),
        ("trial_offsets", _vp),
        ("weights_offsets", _vp),
        ("npoints", _vp),
        ("values", _vp),
        ("dense", _vp),
        ("ld", _i64),
        ("diag_shift", _ct.c_double),
        ("phase_radius", _ct.c_double),
        ("mirror_weights_offset", _i64),
    ]


class PotentialArgs(_ct.Structure):
    _fields_ = [
        ("kernel", _i32),
        ("assembly", _i32),
        ("precision", _i32),
        ("pad0", _i32),
        ("params", _ct.c_double * 4),
        ("grid", GridRec),
        ("space", Space),
        ("nq", _i32),
        ("pad1", _i32),
        ("quad_points", _vp),
        ("quad_weights", _vp),
        ("npoints", _i64),
        ("points", _vp),
        ("coefficients", _vp),
        ("result", _vp),
        ("workspace", _vp),
        ("workspace_bytes", _i64),
        ("phase_radius", _ct.c_double),
    ]


class BatchProblem(_ct.Structure):
    _fields_ = [
        ("grid", GridRec),
        ("support", _vp),
        ("result", _vp),
        ("ld", _i64),
        ("params", _ct.c_double * 4),
        ("phase_radius", _ct.c_double),
        ("precision", _i32),
        ("pad", _i32),
        ("pair_begin", _i64),
        ("pair_count", _i64),
    ]


class BatchArgs(_ct.Structure):
    _fields_ = [
        ("kernel", _i32),
        ("nproblems", _i32),
        ("problems", _ct.POINTER(BatchProblem)),
        ("nq", _i32),
        ("blocks_per_sm", _i32),
        ("quad_points", _vp),
        ("quad_weights", _vp),
        ("npairs", _i64),
        ("test_points", _vp),
        ("trial_points", _vp),
        ("weights", _vp),
        ("test_elements", _vp),
        ("trial_elements", _vp),
        ("test_offsets", _vp),
        ("trial_offsets", _vp),
        ("weights_offsets", _vp),
        ("npoints", _vp),
        ("diag_shift", _ct.c_double),
        ("rows_per_item", _i32),
        ("pad", _i32),
        ("workspace", _vp),
        ("workspace_bytes", _i64),
    ]


BASIS_SCALAR = 0
BASIS_RWG = 1
BASIS_SNC = 2


class IdentityArgs(_ct.Structure):
    _fields_ = [
        ("grid", GridRec),
        ("test", Space),
        ("trial", Space),
        ("test_kind", _i32),
        ("trial_kind", _i32),
        ("nelements", _i64),
        ("elements", _vp),
        ("nq", _i32),
        ("pad", _i32),
        ("quad_points", _vp),
        ("quad_weights", _vp),
        ("rows", _vp),
        ("cols", _vp),
        ("values", _vp),
    ]


class MatmatProblem(_ct.Structure):
    _fields_ = [
        ("a", _vp),
        ("x", _vp),
        ("y", _vp),
        ("rows", _i64),
        ("cols", _i64),
        ("lda", _i64),
        ("ldx", _i64),
        ("ldy", _i64),
    ]


class MatmatArgs(_ct.Structure):
    _fields_ = [
        ("nproblems", _i32),
        ("nrhs", _i32),
        ("problems", _ct.POINTER(MatmatProblem)),
        ("workspace", _vp),
        ("workspace_bytes", _i64),
        ("blocks", _i64),
    ]


class ShapeArgs(_ct.Structure):
    _fields_ = [
        ("grid", GridRec),
        ("normal_mult", _vp),
        ("k", _ct.c_double),
        ("dlp_coeff", _ct.c_double),
        ("eta", _ct.c_double * 2),
        ("deta_dk", _ct.c_double * 2),
        ("identity", _ct.c_double),
        ("nq", _i32),
        ("ndirections", _i32),
        ("quad_points", _vp),
        ("quad_weights", _vp),
        ("npairs", _i64),
        ("test_points", _vp),
        ("trial_points", _vp),
        ("weights", _vp),
        ("test_elements", _vp),
        ("trial_elements", _vp),
        ("test_offsets", _vp),
        ("trial_offsets", _vp),
        ("weights_offsets", _vp),
        ("npoints", _vp),
        ("directions", _vp),
        ("ff_dlp_coeff", _ct.c_double),
        ("ff_eta", _ct.c_double * 2),
        ("ff_deta_dk", _ct.c_double * 2),
        ("incident", _ct.c_double * 3),
        ("rhs_coeff", _ct.c_double * 2),
        ("phi", _vp),
        ("lam", _vp),
        ("u", _vp),
        ("scale_operator", _ct.c_double),
        ("scale_farfield", _ct.c_double),
        ("scale_rhs", _ct.c_double),
        ("vertex_grad", _vp),
        ("k_grad", _vp),
        ("out", _vp),
        ("workspace", _vp),
        ("workspace_bytes", _i64),
        ("phase_radius", _ct.c_double),
    ]


# every exported symbol of include/bemppcuda.h with (restype, argtypes)
SIGNATURES = {
    "bemppcuda_version": (_ct.c_int, []),
    "bemppcuda_last_error": (_ct.c_int, [_ct.c_char_p, _i64]),
    "bemppcuda_grid_geometry": (_ct.c_int, [_vp, _i64, _vp, _i64, _vp, _vp]),
    "bemppcuda_assemble_regular": (_ct.c_int, [_ct.POINTER(RegularArgs), _vp]),
    "bemppcuda_apply_regular": (_ct.c_int, [_ct.POINTER(RegularArgs), _vp, _vp, _vp]),
    "bemppcuda_gemv": (_ct.c_int, [_vp, _i64, _i64, _i64, _vp, _vp, _i32, _vp]),
    "bemppcuda_quadrature_points": (_ct.c_int, [_ct.POINTER(GridRec), _ct.POINTER(Space), _i32, _vp, _vp, _vp, _vp,
                                                _vp]),
    "bemppcuda_project": (_ct.c_int, [_ct.POINTER(GridRec), _ct.POINTER(Space), _i32, _vp, _vp, _vp, _vp, _vp]),
    "bemppcuda_assemble_singular": (_ct.c_int, [_ct.POINTER(SingularArgs), _vp]),
    "bemppcuda_potential_workspace_bytes": (_i64, [_ct.POINTER(PotentialArgs)]),
    "bemppcuda_evaluate_potential": (_ct.c_int, [_ct.POINTER(PotentialArgs), _vp]),
    "bemppcuda_fma_probe": (_ct.c_int, [_i32, _i64, _i64, _vp, _ct.POINTER(_ct.c_double), _vp]),
    "bemppcuda_evaluate_potential_noalloc": (_ct.c_int, [_ct.POINTER(PotentialArgs), _vp]),
    "bemppcuda_batch_workspace_bytes": (_i64, [_i32]),
    "bemppcuda_batch_prepare": (_ct.c_int, [_ct.POINTER(BatchArgs), _vp]),
    "bemppcuda_batch_launch": (_ct.c_int, [_ct.POINTER(BatchArgs), _vp]),
    "bemppcuda_assemble_identity": (_ct.c_int, [_ct.POINTER(IdentityArgs), _vp]),
    "bemppcuda_matmat_workspace_bytes": (_i64, [_i32]),
    "bemppcuda_matmat_prepare": (_ct.c_int, [_ct.POINTER(MatmatArgs), _vp]),
    "bemppcuda_matmat_launch": (_ct.c_int, [_ct.POINTER(MatmatArgs), _vp]),
    "bemppcuda_shape_workspace_bytes": (_i64, [_i64]),
    "bemppcuda_farfield_matrix_dp0": (_ct.c_int, [_ct.POINTER(ShapeArgs), _vp]),
    "bemppcuda_plane_wave_dp0": (_ct.c_int, [_ct.POINTER(ShapeArgs), _vp]),
    "bemppcuda_shape_adjoint_dp0": (_ct.c_int, [_ct.POINTER(ShapeArgs), _vp]),
}

# fixed workspace of bemppcuda_evaluate_potential_noalloc, in doubles
NOALLOC_SCRATCH_DOUBLES = 3 * 1024 * 1024

_lib = None


class BemppCudaError(RuntimeError):
    """A bemppcuda entry point returned a non-zero status."""

    def __init__(self, status, message):
        super().__init__("bemppcuda status %d: %s" % (status, message))
        self.status = status


def load():
    """Load libbemppcuda.so; raise if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libbemppcuda.so not found at %s; build it with `python -m bempp_cuda.build` "
            "(nvcc, sm_100a).  There is no CPU fallback." % LIB_PATH
        )
    lib = _ct.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error():
    buf = _ct.create_string_buffer(1024)
    load().bemppcuda_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status):
    if status != OK:
        raise BemppCudaError(status, last_error())
    return status
