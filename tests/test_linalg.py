"""Device GMRES algorithms, run on CPU torch tensors against numpy solves.

The solver code is plain torch (device-agnostic); on the GPU box the same
functions run on the assembled device matrices (tests/test_gpu_solve.py).
"""

import numpy as np
import pytest
import torch

from bempp_cuda.linalg import gmres_block, gmres_tensor, solve_refined


def _system(n, seed, dtype=torch.complex128):
    rng = np.random.default_rng(seed)
    a = np.eye(n) * 4 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return torch.as_tensor(a).to(dtype), torch.as_tensor(b).to(dtype), a, b


@pytest.mark.parametrize("restart", [5, 30, 200])
def test_gmres_matches_direct_solve(restart):
    A, b, a, bn = _system(120, 1)
    x, info, res, its = gmres_tensor(lambda v: A @ v, b, tol=1e-10, restart=restart, maxiter=2000)
    assert info == 0
    ref = np.linalg.solve(a, bn)
    assert np.linalg.norm(x.numpy() - ref) <= 1e-8 * np.linalg.norm(ref)
    assert res[-1] <= 1e-10 and its > 0


@pytest.mark.parametrize("check_every", [3, 8, 50])
@pytest.mark.parametrize("restart", [7, 200])
def test_deferred_checks_give_the_same_iterate(check_every, restart):
    """Arnoldi steps checked in chunks: same iterate, residual history and count as checking every step
    (the extra steps of the last chunk are discarded); also with a restart length that is not a multiple."""
    A, b, _, _ = _system(120, 9)
    ref = gmres_tensor(lambda v: A @ v, b, tol=1e-10, restart=restart, maxiter=2000)
    got = gmres_tensor(lambda v: A @ v, b, tol=1e-10, restart=restart, maxiter=2000, check_every=check_every)
    assert got[1] == ref[1] == 0 and got[3] == ref[3]
    assert np.allclose(got[2], ref[2], rtol=1e-10, atol=1e-14)
    assert torch.allclose(got[0], ref[0], rtol=1e-12, atol=1e-14)


def test_deferred_checks_respect_maxiter():
    A, b, _, _ = _system(60, 10)
    x, info, res, its = gmres_tensor(lambda v: A @ v, b, tol=1e-30, restart=20, maxiter=13, check_every=5)
    assert info == 13 and its == 13 and len(res) == 14


def test_adjoint_refinement():
    A, b, a, bn = _system(100, 11)
    x, info = solve_refined(A, b, tol=1e-12, inner_tol=1e-4, adjoint=True)
    assert info["converged"]
    ref = np.linalg.solve(a.conj().T, bn)
    assert np.linalg.norm(x.numpy() - ref) <= 1e-10 * np.linalg.norm(ref)


def test_gmres_real_system():
    rng = np.random.default_rng(3)
    a = np.eye(50) * 3 + rng.standard_normal((50, 50)) / 10
    b = rng.standard_normal(50)
    x, info, _, _ = gmres_tensor(lambda v: torch.as_tensor(a) @ v, torch.as_tensor(b), tol=1e-12)
    assert info == 0
    assert np.allclose(x.numpy(), np.linalg.solve(a, b), rtol=1e-9, atol=1e-12)


def test_gmres_zero_rhs():
    A, b, _, _ = _system(10, 2)
    x, info, res, its = gmres_tensor(lambda v: A @ v, torch.zeros_like(b))
    assert info == 0 and its == 0 and float(x.abs().max()) == 0.0


def test_block_gmres_matches_columns():
    A, _, a, _ = _system(80, 4)
    rng = np.random.default_rng(5)
    B = rng.standard_normal((80, 8)) + 1j * rng.standard_normal((80, 8))
    X, infos, iters = gmres_block(lambda V: A @ V, torch.as_tensor(B), tol=1e-10, restart=25)
    assert infos == [0] * 8
    ref = np.linalg.solve(a, B)
    assert np.linalg.norm(X.numpy() - ref) <= 1e-8 * np.linalg.norm(ref)


def test_refinement_reaches_fp64_accuracy():
    A, b, a, bn = _system(150, 6)
    x, info = solve_refined(A, b, tol=1e-12, inner_tol=1e-3)
    assert info["converged"] and info["refinements"] >= 2
    ref = np.linalg.solve(a, bn)
    assert np.linalg.norm(x.numpy() - ref) <= 1e-10 * np.linalg.norm(ref)
