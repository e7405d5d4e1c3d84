"""CUDA path against the oracle and the reference's fixtures (run on a B200).

Tolerances: FP64 path within 1e-12 relative Frobenius of the oracle / live
Numba fixtures, 1e-10 against the legacy golden data (the reference's own test
tolerance); mixed precision within 1e-6 of the FP64 path.
"""

import numpy as np
import pytest

import cases
from conftest import load_golden, probe_vectors, rel_fro

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bempp_cuda import _lib

    _lib.load()


def _gpu_dense(op):
    return op.weak_form().A


@pytest.fixture(scope="module")
def sphere2():
    from bempp_cuda.shapes import regular_sphere

    return regular_sphere(2)


@pytest.mark.parametrize("key", sorted(cases.BOUNDARY))
def test_boundary_matches_oracle(oracle, sphere2, key):
    op, domain, dual = cases.boundary_operator(key, sphere2)
    ref = cases.oracle_dense(oracle, op, domain, dual)
    got = _gpu_dense(op)
    assert got.shape == ref.shape and got.dtype == ref.dtype
    assert rel_fro(got, ref) < 1e-12


NUMBA = load_golden("numba_boundary.npz")


@pytest.mark.parametrize("key", sorted(cases.BOUNDARY))
def test_boundary_matches_live_numba_fixture(key):
    from bempp_cuda.grid import Grid

    grid = Grid(NUMBA["vertices"], NUMBA["elements"])
    op, _, _ = cases.boundary_operator(key, grid)
    assert rel_fro(_gpu_dense(op), NUMBA[key + "__A"]) < 1e-12


LEGACY = load_golden("legacy_boundary.npz")


@pytest.mark.parametrize("key", sorted({k.split("__")[0] for k in LEGACY.files}))
def test_boundary_matches_legacy_golden(sphere_msh_grid, key):
    op, _, _ = cases.boundary_operator(key, sphere_msh_grid)
    mat = _gpu_dense(op)
    rows, cols = LEGACY[key + "__shape"]
    u, w, ii, jj = probe_vectors(rows, cols)
    assert rel_fro(mat @ u, LEGACY[key + "__Au"]) < 1e-10
    assert rel_fro(mat.T @ w, LEGACY[key + "__ATw"]) < 1e-10


@pytest.mark.parametrize("key", ["laplace_slp_p0_p0", "helmholtz_slp_p0_p0", "helmholtz_dlp_p0_p0",
                                 "helmholtz_adlp_p0_p0"])
def test_dp0_level4_matches_oracle(oracle, key):
    """C1-sized DP0 problems (2048 x 2048): the FP64 fast path against the oracle."""
    from bempp_cuda.shapes import regular_sphere

    grid = regular_sphere(4)
    op, domain, dual = cases.boundary_operator(key, grid)
    ref = cases.oracle_dense(oracle, op, domain, dual)
    assert rel_fro(_gpu_dense(op), ref) < 1e-12


def test_dispatcher_regular_and_singular_parts(oracle, sphere2):
    """The reference-interface entry points: regular part into a host result, singular values."""
    from bempp_cuda import cuda_assemblers
    from bempp_cuda.quadrature import SingularPairs, triangle_rule

    for key in ["helmholtz_slp_p1_p1", "maxwell_efie_rwg_snc", "laplace_hyp_p1_p1", "helmholtz_dlp_p0_p0"]:
        op, domain, dual = cases.boundary_operator(key, sphere2)
        d = op.descriptor
        dtype = np.complex128 if d.is_complex else np.float64
        got = np.zeros((dual.global_dof_count, domain.global_dof_count), dtype=dtype)
        cuda_assemblers.dense_assembler("cuda", d, domain, dual, op.parameters, got)
        ref = np.zeros_like(got)
        qp, qw = triangle_rule(4)
        oracle.regular_part(d.kernel_type, d.assembly_type, d.options, domain, dual, qp, qw, ref)
        assert rel_fro(got, ref) < 1e-12, key
        arrays = SingularPairs(sphere2, 4, dual.localised_space.support, domain.localised_space.support).arrays()
        nt, ns = dual.number_of_shape_functions, domain.number_of_shape_functions
        vals = np.zeros(nt * ns * len(arrays[3]), dtype=dtype)
        cuda_assemblers.singular_assembler("cuda", d, sphere2, domain.localised_space, dual.localised_space,
                                           *arrays, d.options, vals)
        _, _, ref_vals = oracle.singular_values(d.kernel_type, d.assembly_type, d.options, domain.localised_space,
                                                dual.localised_space, arrays, d.is_complex)
        assert rel_fro(vals, ref_vals) < 1e-12, key


SINGULAR_VALUE_KEYS = sorted(k for k in cases.BOUNDARY if k.endswith("_p1_p1") or k.endswith("_rwg_snc"))


@pytest.mark.parametrize("key", SINGULAR_VALUE_KEYS)
def test_singular_values_p1_and_rwg(oracle, sphere2, key):
    """Per-pair singular values (the reference interface's flat output, no mirroring) of every P1 x P1 and
    RWG / SNC operator against the oracle: the P1 and Maxwell singular kernels in values mode."""
    from bempp_cuda import cuda_assemblers
    from bempp_cuda.quadrature import SingularPairs

    op, domain, dual = cases.boundary_operator(key, sphere2)
    d = op.descriptor
    dtype = np.complex128 if d.is_complex else np.float64
    arrays = SingularPairs(sphere2, 4, dual.localised_space.support, domain.localised_space.support).arrays()
    nt, ns = dual.number_of_shape_functions, domain.number_of_shape_functions
    vals = np.zeros(nt * ns * len(arrays[3]), dtype=dtype)
    cuda_assemblers.singular_assembler("cuda", d, sphere2, domain.localised_space, dual.localised_space,
                                       *arrays, d.options, vals)
    _, _, ref_vals = oracle.singular_values(d.kernel_type, d.assembly_type, d.options, domain.localised_space,
                                            dual.localised_space, arrays, d.is_complex)
    assert rel_fro(vals, ref_vals) < 1e-12, key


@pytest.mark.parametrize("key", ["helmholtz_slp_p1_p1", "helmholtz_dlp_p1_p1", "helmholtz_hyp_p1_p1",
                                 "maxwell_efie_rwg_snc", "maxwell_mfie_rwg_snc"])
@pytest.mark.parametrize("k", [0.7, 0.9, 12.0])
def test_singular_phase_classes_dense(oracle, sphere2, key, k):
    """Whole matrices (dense singular scatter, vertex pairs mirrored where the kernel allows) in each
    phase class of regular_sphere(2) (2R = 2/3): |k| 2R <= 1/2 (k = 0.7), <= 1 (0.9) and the full
    reduction (12), against the oracle."""
    path, dsp, tsp, _ = cases.BOUNDARY[key]
    from bempp_cuda.space import function_space

    domain, dual = function_space(sphere2, *dsp), function_space(sphere2, *tsp)
    op = cases.resolve("boundary." + path)(domain, domain, dual, k)
    ref = cases.oracle_dense(oracle, op, domain, dual)
    assert rel_fro(_gpu_dense(op), ref) < 1e-12, (key, k)


LEG_POT = load_golden("legacy_potential.npz")
NUM_POT = load_golden("numba_potential.npz")
POT_KEYS = sorted({k.split("__")[0] for k in LEG_POT.files})


@pytest.mark.parametrize("key", POT_KEYS)
def test_potential_matches_fixtures_and_oracle(oracle, sphere_msh_grid, key):
    from bempp_cuda.grid import Grid

    points = LEG_POT[key + "__points"]
    op, space = cases.potential_operator(key, sphere_msh_grid, points)
    got = op.evaluate(LEG_POT[key + "__vec"])
    assert rel_fro(got, LEG_POT[key + "__result"]) < 1e-10
    grid = Grid(NUM_POT["vertices"], NUM_POT["elements"])
    pts = NUM_POT["directions"] if "_ff" in key else NUM_POT["points"]
    op, space = cases.potential_operator(key, grid, pts)
    coeffs = NUM_POT[key + "__coeffs"]
    got = op.evaluate(coeffs)
    assert rel_fro(got, NUM_POT[key + "__result"]) < 1e-12
    assert rel_fro(got, cases.oracle_potential(oracle, op, space, coeffs)) < 1e-12


@pytest.mark.parametrize("name", ["single_layer", "double_layer", "adjoint_double_layer"])
def test_mixed_precision_operator_error(name):
    """FP32 regular pairs: <= 1e-6 relative operator error against the FP64 path (L4, k = 10)."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(4)
    sp = function_space(grid, "DP", 0)
    f = getattr(operators.boundary.helmholtz, name)
    a64 = f(sp, sp, sp, 10.0, device_interface="cuda").weak_form().tensor
    amx = f(sp, sp, sp, 10.0, device_interface="cuda_mixed").weak_form().tensor
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert err < 1e-6, err


def test_invalid_arguments_fail_cleanly():
    """Bad inputs return an error status and leave the context usable."""
    import ctypes

    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream, ptr

    lib = _lib.load()
    verts = torch.zeros((3, 3), dtype=torch.float64, device="cuda")
    verts[1, 0] = 1.0
    verts[2, 1] = 1.0
    elems = torch.tensor([[0, 1, 7]], dtype=torch.int32, device="cuda")  # index 7 out of range
    geom = torch.empty((_lib.GEOM_FIELDS, 1), dtype=torch.float64, device="cuda")
    rc = lib.bemppcuda_grid_geometry(ptr(verts), 3, ptr(elems), 1, ptr(geom), current_stream())
    assert rc == _lib.ERR_INVALID and "out of range" in _lib.last_error()
    rc = lib.bemppcuda_assemble_regular(None, current_stream())
    assert rc == _lib.ERR_INVALID
    args = _lib.RegularArgs()
    args.nq = 99
    args.test.nshape = 1
    args.trial.nshape = 1
    rc = lib.bemppcuda_assemble_regular(ctypes.byref(args), current_stream())
    assert rc == _lib.ERR_INVALID
    torch.cuda.synchronize()
    assert torch.ones(4, device="cuda").sum().item() == 4.0
