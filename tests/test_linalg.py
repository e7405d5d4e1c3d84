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
