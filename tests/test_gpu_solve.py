"""Dense solves on the device: GMRES on assembled operators, mixed-precision refinement."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _plane_wave(k):
    def fun(x, n, domain_index, result):
        result[0] = -np.exp(1j * k * x[2])

    return fun


def _combined(space, k, interface):
    from bempp_cuda import operators

    slp = operators.boundary.helmholtz.single_layer(space, space, space, k, device_interface=interface)
    dlp = operators.boundary.helmholtz.double_layer(space, space, space, k, device_interface=interface)
    ident = operators.boundary.sparse.identity(space, space, space)
    return dlp - 0.5 * ident - 1j * k * slp


def test_fused_combined_field_matches_term_by_term():
    """dlp - 0.5 I - i k slp fused in one pass equals the sum of the separately assembled weak forms."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    k = 7.0
    sp = function_space(regular_sphere(3), "DP", 0)
    fused = _combined(sp, k, "cuda").weak_form().A
    slp = operators.boundary.helmholtz.single_layer(sp, sp, sp, k).weak_form().A
    dlp = operators.boundary.helmholtz.double_layer(sp, sp, sp, k).weak_form().A
    ref = dlp - 0.5 * np.diag(sp.grid.volumes) - 1j * k * slp
    assert np.linalg.norm(fused - ref) <= 1e-12 * np.linalg.norm(ref)


def test_device_gmres_matches_direct_solve():
    from bempp_cuda.grid_function import GridFunction
    from bempp_cuda.linalg import gmres
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    k = 5.0
    sp = function_space(regular_sphere(3), "DP", 0)
    lhs = _combined(sp, k, "cuda")
    rhs = GridFunction(sp, fun=_plane_wave(k))
    sol, info, its = gmres(lhs, rhs, tol=1e-10, return_iteration_count=True)
    assert info == 0 and its > 0
    a = lhs.weak_form().A
    ref = np.linalg.solve(a, rhs.projections(sp))
    assert np.linalg.norm(sol.coefficients - ref) <= 1e-8 * np.linalg.norm(ref)


def test_mixed_refinement_matches_fp64_solve():
    """Mixed-precision assembly + refinement with FP64 residuals (the FP64 operator evaluated
    matrix-free) against the FP64 solve (L4, k = 10): within 1e-8, the bound of the benchmark's
    precision configuration; residuals with the mixed matrix instead stop at its own solution."""
    from bempp_cuda.grid_function import GridFunction
    from bempp_cuda.linalg import gmres_tensor, solve_refined
    from bempp_cuda.operators import fp64_matvec
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    k = 10.0
    sp = function_space(regular_sphere(4), "DP", 0)
    a64 = _combined(sp, k, "cuda").weak_form().tensor
    opmx = _combined(sp, k, "cuda_mixed")
    amx = opmx.weak_form().tensor
    op_err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert op_err < 1e-6
    b = torch.as_tensor(GridFunction(sp, fun=_plane_wave(k)).projections(sp), device="cuda")
    x64, info, _, _ = gmres_tensor(lambda v: torch.mv(a64, v), b, tol=1e-12, restart=200)
    assert info == 0
    xmx, rinfo = solve_refined(amx, b, tol=1e-10, inner_tol=1e-4, residual=fp64_matvec(opmx, amx))
    assert rinfo["converged"]
    diff = (torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64)).item()
    assert diff < 1e-8, (diff, op_err)
    # residuals with the mixed matrix converge to the mixed operator's solution instead
    xm2, _ = solve_refined(amx, b, tol=1e-10, inner_tol=1e-4)
    diff_mixed = (torch.linalg.norm(xm2 - x64) / torch.linalg.norm(x64)).item()
    assert diff < diff_mixed


def test_block_gmres_eight_rhs_on_device():
    from bempp_cuda.linalg import gmres_block
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    sp = function_space(regular_sphere(3), "DP", 0)
    a = _combined(sp, 4.0, "cuda").weak_form().tensor
    rng = np.random.default_rng(8)
    B = torch.as_tensor(rng.standard_normal((a.shape[0], 8)) + 1j * rng.standard_normal((a.shape[0], 8)),
                        device="cuda")
    X, infos, iters = gmres_block(lambda V: a @ V, B, tol=1e-9, restart=60)
    assert infos == [0] * 8
    assert (torch.linalg.norm(a @ X - B) / torch.linalg.norm(B)).item() < 1e-8


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64, torch.float64])
@pytest.mark.parametrize("restart", [10, 200])
def test_graph_arnoldi_matches_host_driven_gmres(dtype, restart):
    """Arnoldi steps replayed from one CUDA graph (checked every 7 steps) = the step-by-step loop, with
    restarts, for complex and real systems; and the adjoint through the transposed view."""
    from bempp_cuda.linalg import adjoint_matvec, gmres_tensor

    rng = np.random.default_rng(12)
    n = 300
    a = np.eye(n) * 4 + rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal(n)
    if dtype.is_complex:
        a = a + 1j * rng.standard_normal((n, n)) / np.sqrt(n)
        b = b + 1j * rng.standard_normal(n)
    A = torch.as_tensor(a, device="cuda").to(dtype)
    bt = torch.as_tensor(b, device="cuda").to(dtype)
    tol = 1e-5 if dtype == torch.complex64 else 1e-11
    ref = gmres_tensor(lambda v: torch.mv(A, v), bt, tol=tol, restart=restart, maxiter=3000)
    got = gmres_tensor(lambda v: torch.mv(A, v), bt, tol=tol, restart=restart, maxiter=3000, check_every=7,
                       graph=True)
    assert got[1] == ref[1] == 0 and got[3] == ref[3]
    rtol = 1e-4 if dtype == torch.complex64 else 1e-9
    assert torch.allclose(got[0], ref[0], rtol=rtol, atol=rtol * float(ref[0].abs().max()))
    if dtype == torch.complex128:
        adj = gmres_tensor(adjoint_matvec(A), bt, tol=1e-11, restart=restart, maxiter=3000, check_every=7, graph=True)
        x = np.linalg.solve(a.conj().T, b)
        assert adj[1] == 0
        assert np.linalg.norm(adj[0].cpu().numpy() - x) <= 1e-9 * np.linalg.norm(x)
