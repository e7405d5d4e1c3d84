"""Pin the CPU oracle to the reference: its golden matrices and live Numba outputs."""

import numpy as np
import pytest

import cases
from conftest import load_golden, probe_vectors, rel_fro

LEGACY = load_golden("legacy_boundary.npz")
LEGACY_KEYS = sorted({k.split("__")[0] for k in LEGACY.files})


@pytest.mark.parametrize("key", LEGACY_KEYS)
def test_oracle_matches_legacy_golden(oracle, sphere_msh_grid, key):
    """Reference test data test/data/*_boundary*.npy, tolerance of the reference tests (1e-10)."""
    op, domain, dual = cases.boundary_operator(key, sphere_msh_grid)
    mat = cases.oracle_dense(oracle, op, domain, dual)
    rows, cols = LEGACY[key + "__shape"]
    assert mat.shape == (rows, cols)
    u, w, ii, jj = probe_vectors(rows, cols)
    assert rel_fro(mat @ u, LEGACY[key + "__Au"]) < 1e-10
    assert rel_fro(mat.T @ w, LEGACY[key + "__ATw"]) < 1e-10
    assert abs(np.linalg.norm(mat) - LEGACY[key + "__fro"]) < 1e-10 * LEGACY[key + "__fro"]
    assert np.allclose(mat[ii, jj], LEGACY[key + "__entries"], rtol=1e-10, atol=1e-14 * LEGACY[key + "__fro"])


NUMBA = load_golden("numba_boundary.npz")


@pytest.mark.parametrize("key", sorted(cases.BOUNDARY))
def test_oracle_matches_live_numba(oracle, key):
    """Full matrices of the reference Numba path on regular_sphere(1): 1e-12 relative Frobenius."""
    from bempp_cuda.grid import Grid

    grid = Grid(NUMBA["vertices"], NUMBA["elements"])
    op, domain, dual = cases.boundary_operator(key, grid)
    ref = NUMBA[key + "__A"]
    assert list(NUMBA[key + "__desc"]) == [op.descriptor.kernel_type, op.descriptor.assembly_type]
    assert np.allclose(NUMBA[key + "__options"], op.descriptor.options)
    mat = cases.oracle_dense(oracle, op, domain, dual)
    assert rel_fro(mat, ref) < 1e-12


LEG_POT = load_golden("legacy_potential.npz")
POT_KEYS = sorted({k.split("__")[0] for k in LEG_POT.files})


@pytest.mark.parametrize("key", POT_KEYS)
def test_oracle_potential_matches_legacy(oracle, sphere_msh_grid, key):
    points = LEG_POT[key + "__points"]
    op, space = cases.potential_operator(key, sphere_msh_grid, points)
    res = cases.oracle_potential(oracle, op, space, LEG_POT[key + "__vec"])
    ref = LEG_POT[key + "__result"]
    assert rel_fro(res, ref) < 1e-10


NUM_POT = load_golden("numba_potential.npz")


@pytest.mark.parametrize("key", POT_KEYS)
def test_oracle_potential_matches_live_numba(oracle, key):
    from bempp_cuda.grid import Grid

    grid = Grid(NUM_POT["vertices"], NUM_POT["elements"])
    pts = NUM_POT["directions"] if "_ff" in key else NUM_POT["points"]
    op, space = cases.potential_operator(key, grid, pts)
    res = cases.oracle_potential(oracle, op, space, NUM_POT[key + "__coeffs"])
    assert rel_fro(res, NUM_POT[key + "__result"]) < 1e-12
