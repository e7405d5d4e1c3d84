"""Symmetric DP0 sweep (A_ij and A_ji from one pass) against per-entry evaluation (run on a B200)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


KERNELS = [
    ("laplace_single_layer", []),
    ("laplace_double_layer", []),
    ("laplace_adjoint_double_layer", []),
    ("helmholtz_single_layer", [4.0, 0.0]),
    ("helmholtz_double_layer", [4.0, 0.0]),
    ("helmholtz_adjoint_double_layer", [4.0, 0.0]),
    ("helmholtz_combined_field", [7.0, 0.0, 0.0, -7.0]),
    ("helmholtz_combined_field", [40.0, 0.0, 1.5, -40.0]),  # |k| (R_i + R_j) > 1: reduced phase
    # complex wavenumbers: the FP64 sweep as phase class 3, the mixed sweep with the amplitude e^{-beta r'}
    # split about the centroids (the last case: |k| (R_i + R_j) > 1 and a strong damping)
    ("helmholtz_single_layer", [4.0, 0.7]),
    ("helmholtz_double_layer", [4.0, 0.7]),
    ("helmholtz_adjoint_double_layer", [4.0, 0.7]),
    ("helmholtz_combined_field", [7.0, 0.5, 0.0, -7.0]),
    ("helmholtz_combined_field", [30.0, 9.0, 1.0, -30.0]),
    # modified Helmholtz (real kernel; both sweeps, the mixed one with e^{-r'} split about the centroids)
    ("modified_helmholtz_single_layer", [2.0]),
    ("modified_helmholtz_double_layer", [2.0]),
    ("modified_helmholtz_adjoint_double_layer", [6.0]),
    ("modified_helmholtz_double_layer", [25.0]),
]


def _assemble(grid, kernel, options, precision, symmetric):
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import OperatorDescriptor, Parameters
    from bempp_cuda.space import function_space

    sp = function_space(grid, "DP", 0)
    is_complex = kernel.startswith("helmholtz")
    desc = OperatorDescriptor("probe", options, kernel, "default_scalar", "double", is_complex, None, 1)
    n = grid.number_of_elements
    out = torch.full((n, n), float("nan"), dtype=torch.complex128 if is_complex else torch.float64, device="cuda")
    regular_into(out, desc, sp, sp, Parameters(), precision=precision, overwrite=True, symmetric=symmetric)
    singular_into_dense(out, desc, sp, sp, Parameters())
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("kernel,options", KERNELS)
def test_symmetric_sweep_matches_entrywise(kernel, options):
    from bempp_cuda import _lib
    from bempp_cuda.shapes import ellipsoid

    grid = ellipsoid(3, 1.0, 0.8, 1.2)  # 512 elements: partial column block and diagonal tiles
    sym64 = _assemble(grid, kernel, options, _lib.FP64, True)
    ref64 = _assemble(grid, kernel, options, _lib.FP64, False)
    assert torch.isfinite(torch.view_as_real(sym64) if sym64.is_complex() else sym64).all()
    assert (torch.linalg.norm(sym64 - ref64) / torch.linalg.norm(ref64)).item() < 1e-13
    symmx = _assemble(grid, kernel, options, _lib.MIXED, True)
    refmx = _assemble(grid, kernel, options, _lib.MIXED, False)
    assert (torch.linalg.norm(symmx - ref64) / torch.linalg.norm(ref64)).item() < 1e-6
    assert (torch.linalg.norm(refmx - ref64) / torch.linalg.norm(ref64)).item() < 1e-6


def test_symmetric_sweep_odd_size():
    """300 elements of a 512-element grid would break the square check; use a full odd grid instead."""
    from bempp_cuda import _lib
    from bempp_cuda.grid import Grid
    from bempp_cuda.shapes import regular_sphere

    g = regular_sphere(3)
    keep = np.arange(g.number_of_elements - 37)  # open surface, ragged last column block
    used = np.unique(g.elements[:, keep])
    remap = -np.ones(g.vertices.shape[1], dtype=np.int64)
    remap[used] = np.arange(len(used))
    grid = Grid(g.vertices[:, used], remap[g.elements[:, keep]].astype(np.uint32))
    for kernel, options in (("helmholtz_combined_field", [5.0, 0.0, 0.0, -5.0]), ("laplace_double_layer", [])):
        a = _assemble(grid, kernel, options, _lib.FP64, True)
        b = _assemble(grid, kernel, options, _lib.FP64, False)
        assert (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item() < 1e-13


@pytest.mark.parametrize("path,k", [("laplace.single_layer", None), ("helmholtz.single_layer", 4.0),
                                    ("laplace.hypersingular", None), ("helmholtz.hypersingular", 4.0),
                                    ("laplace.double_layer", None), ("laplace.adjoint_double_layer", None),
                                    ("helmholtz.double_layer", 2.0), ("helmholtz.double_layer", 4.0),
                                    ("helmholtz.double_layer", 40.0), ("helmholtz.adjoint_double_layer", 4.0),
                                    ("helmholtz.single_layer", 3.0 + 0.5j), ("helmholtz.double_layer", 3.0 + 0.5j),
                                    ("helmholtz.adjoint_double_layer", 3.0 + 0.5j),
                                    ("helmholtz.hypersingular", 3.0 + 0.5j)])
def test_p1_symmetric_sweep_matches_entrywise(path, k):
    """P1 operators: the symmetric sweep against per-pair evaluation.

    Single layer and hypersingular add each block at (i, j) and its transpose;
    the double and adjoint double layer form the transposed pair's own block
    from the other element's normal.  k = 2, 4, 40 reach the three phase
    classes (|k| (R_i + R_j) <= 1/2, <= 1, reduced); k = 3 + 0.5i the complex
    wavenumber class (exp(-Im k r) per point pair).
    """
    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "P", 1)
    f = operators.boundary
    for part in path.split("."):
        f = getattr(f, part)
    op = f(sp, sp, sp) if k is None else f(sp, sp, sp, k)
    d = op.descriptor
    n = sp.global_dof_count
    dtype = torch.complex128 if d.is_complex else torch.float64
    out = []
    # symmetric (both blocks by atomics), per pair, and symmetric into a zeroed
    # result (blocks of i < j, then A = U + U^T for single layer / hypersingular)
    for sym, zero in ((True, False), (False, False), (True, True)):
        a = torch.zeros((n, n), dtype=dtype, device="cuda")
        regular_into(a, d, sp, sp, Parameters(), symmetric=sym, result_is_zero=zero)
        singular_into_dense(a, d, sp, sp, Parameters())
        out.append(a)
    torch.cuda.synchronize()
    assert (torch.linalg.norm(out[0] - out[1]) / torch.linalg.norm(out[1])).item() < 1e-13
    assert (torch.linalg.norm(out[2] - out[1]) / torch.linalg.norm(out[1])).item() < 1e-13
    # accumulating into a matrix that already holds values (no zero promise): prior + A
    prior = torch.randn((n, n), dtype=dtype, device="cuda")
    acc = prior.clone()
    regular_into(acc, d, sp, sp, Parameters())
    singular_into_dense(acc, d, sp, sp, Parameters())
    scale = (torch.linalg.norm(prior) + torch.linalg.norm(out[1])).item()
    assert torch.linalg.norm(acc - prior - out[1]).item() < 1e-13 * scale


@pytest.mark.parametrize("name", ["electric_field", "magnetic_field"])
@pytest.mark.parametrize("k", [1.0, 3.0, 20.0, 3.0 + 0.5j, 1.0 + 2.0j])
def test_maxwell_rwg_kernel_against_oracle(oracle, name, k):
    """Maxwell EFIE / MFIE (RWG domain, SNC dual) through the RWG kernel: the
    symmetric sweep (RWG and SNC share their dof maps) and the per-pair sweep
    against the oracle.  k = 1, 3, 20 on a 512-element ellipsoid reach the
    three phase classes; 3 + 0.5i and 1 + 2i the complex wavenumber class."""
    from cases import oracle_dense

    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    rwg = function_space(grid, "RWG", 0)
    snc = function_space(grid, "SNC", 0)
    op = getattr(operators.boundary.maxwell, name)(rwg, rwg, snc, k)
    ref = oracle_dense(oracle, op, rwg, snc)
    d = op.descriptor
    n = rwg.global_dof_count
    for sym in (True, False):
        a = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
        regular_into(a, d, rwg, snc, Parameters(), symmetric=sym)
        singular_into_dense(a, d, rwg, snc, Parameters())
        got = a.cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (name, k, sym)


@pytest.mark.parametrize("name", ["single_layer", "double_layer", "adjoint_double_layer"])
@pytest.mark.parametrize("k", [3.0 + 0.5j, 1.0 + 2.0j])
def test_dp0_complex_wavenumber_against_oracle(oracle, name, k):
    """DP0 Helmholtz operators with a complex wavenumber: symmetric sweep and per-pair evaluation against the
    oracle."""
    from cases import oracle_dense

    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "DP", 0)
    op = getattr(operators.boundary.helmholtz, name)(sp, sp, sp, k)
    ref = oracle_dense(oracle, op, sp, sp)
    d = op.descriptor
    n = sp.global_dof_count
    for sym in (True, False):
        a = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
        regular_into(a, d, sp, sp, Parameters(), symmetric=sym)
        singular_into_dense(a, d, sp, sp, Parameters())
        got = a.cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (name, k, sym)


@pytest.mark.parametrize("name", ["single_layer", "double_layer", "adjoint_double_layer"])
@pytest.mark.parametrize("omega", [1.5, 5.0])
def test_dp0_modified_helmholtz_against_oracle(oracle, name, omega):
    """DP0 modified Helmholtz: symmetric sweep and per-pair evaluation, DP0 singular routine, against the oracle."""
    from cases import oracle_dense

    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "DP", 0)
    op = getattr(operators.boundary.modified_helmholtz, name)(sp, sp, sp, omega)
    ref = oracle_dense(oracle, op, sp, sp)
    d = op.descriptor
    n = sp.global_dof_count
    for sym in (True, False):
        a = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        regular_into(a, d, sp, sp, Parameters(), symmetric=sym)
        singular_into_dense(a, d, sp, sp, Parameters())
        got = a.cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (name, omega, sym)


@pytest.mark.parametrize("name", ["single_layer", "double_layer", "adjoint_double_layer", "hypersingular"])
@pytest.mark.parametrize("omega", [1.5, 6.0])
def test_modified_helmholtz_p1_kernel_against_oracle(oracle, name, omega):
    """Modified Helmholtz (real kernel exp(-w r) / (4 pi r)) on P1 through regular_p1: the symmetric / skew
    sweep, its deferred transpose and the per-pair sweep against the oracle."""
    from cases import oracle_dense

    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "P", 1)
    op = getattr(operators.boundary.modified_helmholtz, name)(sp, sp, sp, omega)
    ref = oracle_dense(oracle, op, sp, sp)
    d = op.descriptor
    n = sp.global_dof_count
    assert not d.is_complex
    for sym, zero in ((True, False), (False, False), (True, True)):
        a = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        regular_into(a, d, sp, sp, Parameters(), symmetric=sym, result_is_zero=zero)
        singular_into_dense(a, d, sp, sp, Parameters())
        got = a.cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (name, omega, sym, zero)


@pytest.mark.parametrize("kernel,options", KERNELS)
def test_singular_vertex_pairs_mirrored(kernel, options):
    """DP0 singular pass: each vertex-adjacent pair evaluated once for both orders = every ordered pair."""
    from bempp_cuda.assembly import singular_into_dense
    from bempp_cuda.operators import OperatorDescriptor, Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.0, 0.8, 1.2)
    sp = function_space(grid, "DP", 0)
    is_complex = kernel.startswith("helmholtz")
    desc = OperatorDescriptor("probe", options, kernel, "default_scalar", "double", is_complex, None, 1)
    n = grid.number_of_elements
    out = []
    for mirror in (True, False):
        a = torch.zeros((n, n), dtype=torch.complex128 if is_complex else torch.float64, device="cuda")
        singular_into_dense(a, desc, sp, sp, Parameters(), diag_shift=-0.5, mirror=mirror)
        out.append(a)
    torch.cuda.synchronize()
    assert (torch.linalg.norm(out[0] - out[1]) / torch.linalg.norm(out[1])).item() < 1e-13


@pytest.mark.parametrize("blocks", [1, 5, 16])
def test_weak_form_to_host_streams_row_blocks(blocks):
    """Row-block symmetric assembly streamed to pinned host memory = the device weak form."""
    from bempp_cuda import operators

    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.0, 0.8, 1.2)
    sp = function_space(grid, "DP", 0)
    k = 6.0
    for interface, tol in (("cuda", 1e-14), ("cuda_mixed", 1e-14)):
        slp = operators.boundary.helmholtz.single_layer(sp, sp, sp, k, device_interface=interface)
        dlp = operators.boundary.helmholtz.double_layer(sp, sp, sp, k, device_interface=interface)
        ident = operators.boundary.sparse.identity(sp, sp, sp, device_interface=interface)
        lhs = dlp - 0.5 * ident - 1j * k * slp
        host = operators.weak_form_to_host(lhs, blocks=blocks)
        assert host.is_pinned()
        ref = lhs.weak_form().tensor.cpu()
        assert (torch.linalg.norm(host - ref) / torch.linalg.norm(ref)).item() < tol
    # a plain DP0 operator and a P1 operator (assembled whole, then copied)
    for space in (sp, function_space(grid, "P", 1)):
        op = operators.boundary.laplace.double_layer(space, space, space)
        host = operators.weak_form_to_host(op, blocks=blocks)
        ref = op.weak_form().tensor.cpu()
        assert (torch.linalg.norm(host - ref) / torch.linalg.norm(ref)).item() < 1e-14


def test_weak_form_to_host_on_a_row_block():
    """A row block of the combined field (dual restricted to some elements, as one rank assembles it)."""
    import numpy as np

    from bempp_cuda import operators
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.0, 0.8, 1.2)
    d = function_space(grid, "DP", 0)
    t = function_space(grid, "DP", 0, support_elements=np.arange(100, 300))
    k = 5.0
    slp = operators.boundary.helmholtz.single_layer(d, d, t, k)
    dlp = operators.boundary.helmholtz.double_layer(d, d, t, k)
    ident = operators.boundary.sparse.identity(d, d, t)
    full_slp = operators.boundary.helmholtz.single_layer(d, d, d, k)
    full_dlp = operators.boundary.helmholtz.double_layer(d, d, d, k)
    full_id = operators.boundary.sparse.identity(d, d, d)
    host = operators.weak_form_to_host(dlp - 0.5 * ident - 1j * k * slp)
    ref = (full_dlp - 0.5 * full_id - 1j * k * full_slp).weak_form().tensor.cpu()[100:300]
    assert host.shape == (200, grid.number_of_elements)
    assert (torch.linalg.norm(host - ref) / torch.linalg.norm(ref)).item() < 1e-13


@pytest.mark.parametrize("world", [1, 3])
def test_row_blocks_reproduce_the_operator(world):
    """distributed.assemble_row_block: each rank's rows (a DP0 dual restricted to its block; its
    singular pairs) equal those rows of the whole operator, identity shift included."""
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.distributed import assemble_row_block, row_block
    from bempp_cuda.operators import OperatorDescriptor, Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    sp = function_space(grid, "DP", 0)
    desc = OperatorDescriptor("probe", [6.0, 0.0, 0.0, -6.0], "helmholtz_combined_field", "default_scalar", "double",
                              True, None, 1)
    n = grid.number_of_elements
    full = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    regular_into(full, desc, sp, sp, Parameters(), overwrite=True)
    singular_into_dense(full, desc, sp, sp, Parameters(), diag_shift=-0.5)
    for rank in range(world):
        lo, hi = row_block(n, world, rank)
        for precision, tol in ((None, 1e-13), (_lib.MIXED, 1e-6)):
            block = assemble_row_block(grid, desc, world, rank, precision=precision, diag_shift=-0.5)
            assert block.shape == (hi - lo, n)
            ref = full[lo:hi]
            assert (torch.linalg.norm(block - ref) / torch.linalg.norm(ref)).item() < tol, (rank, precision)
