"""The sparse L2 identity (csrc/identity.cu) against the reference (run on a B200).

Fixtures (tests/golden/identity.npz, written by make_golden.py from the
reference): its own golden test/data/sparse_identity_*.npy on sphere.msh
(P0 / P1 pairs and RWG -> SNC, compared there with rtol 1e-10 and atol 1e-14
for SNC / RWG) and the live reference Numba path on regular_sphere(2) for DP1,
P1 / DP1, RWG / RWG, SNC / SNC and SNC -> RWG.  Tolerance here: 1e-13
relative Frobenius norm and 1e-14 absolute per entry.
"""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

ID = load_golden("identity.npz")
SPACES = {
    "p0_p0": (("DP", 0), ("DP", 0)),
    "p1_p1": (("P", 1), ("P", 1)),
    "p0_p1": (("P", 1), ("DP", 0)),
    "p1_p0": (("DP", 0), ("P", 1)),
    "snc_rwg": (("RWG", 0), ("SNC", 0)),
    "dp1_dp1": (("DP", 1), ("DP", 1)),
    "p1_dp1": (("DP", 1), ("P", 1)),
    "rwg_rwg": (("RWG", 0), ("RWG", 0)),
    "snc_snc": (("SNC", 0), ("SNC", 0)),
    "rwg_snc": (("SNC", 0), ("RWG", 0)),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _golden(prefix):
    rows, cols = ID[prefix + "__rows"], ID[prefix + "__cols"]
    out = np.zeros(tuple(ID[prefix + "__shape"]))
    out[rows, cols] = ID[prefix + "__vals"]
    return out


def _dense(weak):
    from bempp_cuda.operators import DiagonalOperator

    if isinstance(weak, DiagonalOperator):
        return torch.diag(weak.values).cpu().numpy()
    return weak.to_dense()


def _identity(grid, key):
    from bempp_cuda import operators
    from bempp_cuda.space import function_space

    dsp, tsp = SPACES[key]
    d = function_space(grid, *dsp)
    t = function_space(grid, *tsp)
    return operators.boundary.sparse.identity(d, d, t), d, t


def _close(got, ref):
    assert got.shape == ref.shape
    assert np.linalg.norm(got - ref) <= 1e-13 * np.linalg.norm(ref)
    assert np.max(np.abs(got - ref)) <= 1e-14


@pytest.mark.parametrize("key", sorted(k.split("__")[0][len("legacy_"):] for k in ID.files
                                       if k.startswith("legacy_") and k.endswith("__shape")))
def test_identity_matches_reference_golden(sphere_msh_grid, key):
    op, _, _ = _identity(sphere_msh_grid, key)
    _close(_dense(op.weak_form()), _golden("legacy_" + key))


@pytest.mark.parametrize("key", sorted(k.split("__")[0][len("live_"):] for k in ID.files
                                       if k.startswith("live_") and k.endswith("__shape")))
def test_identity_matches_live_reference(key):
    from bempp_cuda.grid import Grid

    grid = Grid(ID["vertices"], ID["elements"])
    op, _, _ = _identity(grid, key)
    _close(_dense(op.weak_form()), _golden("live_" + key))


def test_sparse_products_and_algebra():
    """Matvec, scaling and sums of the sparse weak form against its dense matrix."""
    from bempp_cuda.grid import Grid

    grid = Grid(ID["vertices"], ID["elements"])
    op, d, t = _identity(grid, "p1_dp1")
    w = op.weak_form()
    dense = _dense(w)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(d.global_dof_count) + 1j * rng.standard_normal(d.global_dof_count)
    assert np.allclose(w @ x, dense @ x, rtol=1e-13, atol=1e-15)
    xt = torch.as_tensor(x.real, device="cuda")
    assert np.allclose((w @ xt).cpu().numpy(), dense @ x.real, rtol=1e-13, atol=1e-15)
    assert np.allclose(_dense((-2.5) * w), -2.5 * dense)
    assert np.allclose(_dense(w + w * 1j), (1 + 1j) * dense)
    assert np.allclose(_dense(w - w), 0.0)


@pytest.mark.parametrize("case", ["laplace_p1", "maxwell_rwg_snc"])
def test_dense_plus_identity(case):
    """Second-kind operators with a non-DP0 identity: K - 1/2 I assembled on the device."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(2)
    if case == "laplace_p1":
        sp = function_space(grid, "P", 1)
        k_op = operators.boundary.laplace.double_layer(sp, sp, sp)
        ident = operators.boundary.sparse.identity(sp, sp, sp)
    else:
        rwg = function_space(grid, "RWG", 0)
        snc = function_space(grid, "SNC", 0)
        k_op = operators.boundary.maxwell.magnetic_field(rwg, rwg, snc, 2.0)
        ident = operators.boundary.sparse.identity(rwg, rwg, snc)
    combined = (k_op - 0.5 * ident).weak_form()
    ref = k_op.weak_form().A - 0.5 * _dense(ident.weak_form())
    got = combined.A
    assert np.linalg.norm(got - ref) <= 1e-14 * np.linalg.norm(ref)
    host = operators.weak_form_to_host(k_op - 0.5 * ident)
    assert np.array_equal(host.numpy(), got)
    swapped = (-0.5 * ident + k_op).weak_form().A
    assert np.linalg.norm(swapped - ref) <= 1e-14 * np.linalg.norm(ref)


def test_identity_rejects_mixed_scalar_and_vector_spaces():
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(1)
    p1 = function_space(grid, "P", 1)
    rwg = function_space(grid, "RWG", 0)
    with pytest.raises(ValueError, match="two scalar spaces"):
        operators.boundary.sparse.identity(p1, p1, rwg).weak_form()
