"""Mixed precision on P1 spaces (run on a B200).

The single layer, double layer, adjoint double layer and hypersingular
operators on P1 -- Helmholtz (real and complex k), Laplace and modified
Helmholtz -- evaluate their regular pairs in FP32 (``regular_p1_mixed``) under
``device_interface="cuda_mixed"``; their operator error against the FP64 path
and the oracle is held to the mixed-precision bound (1e-6 relative
Frobenius); so do a P1 space beside a DP0 one and the Maxwell electric and
magnetic fields on RWG / SNC (real and complex k).  Operators without a
mixed kernel (Re k <= 0) run in FP64 under the same interface.
"""

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _op(path, sp, k, interface):
    from bempp_cuda import operators

    f = operators.boundary
    for part in path.split("."):
        f = getattr(f, part)
    return f(sp, sp, sp, device_interface=interface) if k is None else f(sp, sp, sp, k, device_interface=interface)


@pytest.mark.parametrize("k", [2.0, 4.0, 40.0])
@pytest.mark.parametrize("path", ["helmholtz.single_layer", "helmholtz.hypersingular", "helmholtz.double_layer",
                                  "helmholtz.adjoint_double_layer"])
def test_mixed_p1_against_fp64_and_oracle(oracle, path, k):
    """k = 2, 4, 40 on a 512-element ellipsoid reach the three phase classes."""
    from cases import oracle_dense

    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "P", 1)
    a64 = _op(path, sp, k, "cuda").weak_form().tensor
    amx = _op(path, sp, k, "cuda_mixed").weak_form().tensor
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err  # FP32 evaluation: close, not identical
    ref = oracle_dense(oracle, _op(path, sp, k, "cuda"), sp, sp)
    assert rel_fro(amx.cpu().numpy(), ref) < 1e-6


OPS = ["single_layer", "hypersingular", "double_layer", "adjoint_double_layer"]
# (family, parameter): complex wavenumbers in the three phase classes of Re k, modified Helmholtz at a small
# and a large omega, Laplace
FAMILIES = [("laplace", None), ("modified_helmholtz", 1.5), ("modified_helmholtz", 12.0),
            ("helmholtz", 2.0 + 0.5j), ("helmholtz", 4.0 + 1.0j), ("helmholtz", 40.0 + 2.0j)]


@pytest.mark.parametrize("family,k", FAMILIES)
@pytest.mark.parametrize("name", OPS)
def test_mixed_p1_other_kernels_against_fp64_and_oracle(oracle, family, name, k):
    """Laplace, modified Helmholtz and complex-k Helmholtz on a 512-element ellipsoid: FP32 pairs within 1e-6
    of the FP64 weak form and of the oracle; real kernels give real matrices."""
    from cases import oracle_dense

    from bempp_cuda import assembly
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    sp = function_space(grid, "P", 1)
    path = family + "." + name
    a64 = _op(path, sp, k, "cuda").weak_form().tensor
    assembly.FP64_FALLBACKS.clear()
    amx = _op(path, sp, k, "cuda_mixed").weak_form().tensor
    assert not assembly.FP64_FALLBACKS  # a mixed kernel ran
    assert amx.dtype == a64.dtype == (torch.complex128 if family == "helmholtz" else torch.float64)
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err
    ref = oracle_dense(oracle, _op(path, sp, k, "cuda"), sp, sp)
    assert rel_fro(amx.cpu().numpy(), ref) < 1e-6


@pytest.mark.parametrize("family,k", [("helmholtz", 5.0), ("helmholtz", 5.0 + 1.0j), ("laplace", None),
                                      ("modified_helmholtz", 3.0)])
@pytest.mark.parametrize("name", OPS)
def test_mixed_p1_sweeps_agree(family, name, k):
    """Symmetric sweep (both blocks by atomics, U + U^T into a zeroed result, or for the double layers the
    skew sweep) and per-pair sweep."""
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    sp = function_space(grid, "P", 1)
    d = _op(family + "." + name, sp, k, "cuda").descriptor
    n = sp.global_dof_count
    dtype = torch.complex128 if family == "helmholtz" else torch.float64
    out = {}
    for precision in (_lib.FP64, _lib.MIXED):
        for sym, zero in ((True, False), (False, False), (True, True)):
            a = torch.zeros((n, n), dtype=dtype, device="cuda")
            regular_into(a, d, sp, sp, Parameters(), precision=precision, symmetric=sym, result_is_zero=zero)
            singular_into_dense(a, d, sp, sp, Parameters())
            out[(precision, sym, zero)] = a
    ref = out[(_lib.FP64, False, False)]
    for key, a in out.items():
        tol = 1e-13 if key[0] == _lib.FP64 else 1e-6
        assert (torch.linalg.norm(a - ref) / torch.linalg.norm(ref)).item() < tol, key


@pytest.mark.parametrize("path,k", [("laplace.double_layer", None), ("helmholtz.single_layer", 3.0 + 0.5j),
                                    ("helmholtz.adjoint_double_layer", 4.0), ("modified_helmholtz.single_layer", 2.0)])
@pytest.mark.parametrize("p1_side", ["domain", "dual"])
def test_mixed_p1_p0_pairs(oracle, path, k, p1_side):
    """A P1 space beside a DP0 one (either side): the mixed P1 kernel with the P0 side's constant function,
    within 1e-6 of FP64 and of the oracle."""
    from cases import oracle_dense

    from bempp_cuda import assembly, operators
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    p1, dp0 = function_space(grid, "P", 1), function_space(grid, "DP", 0)
    dom, dual = (p1, dp0) if p1_side == "domain" else (dp0, p1)
    f = operators.boundary
    for part in path.split("."):
        f = getattr(f, part)
    args = (dom, dom, dual) if k is None else (dom, dom, dual, k)
    op64 = f(*args, device_interface="cuda")
    a64 = op64.weak_form().tensor
    assembly.FP64_FALLBACKS.clear()
    amx = f(*args, device_interface="cuda_mixed").weak_form().tensor
    assert not assembly.FP64_FALLBACKS  # a mixed kernel ran
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err
    assert rel_fro(amx.cpu().numpy(), oracle_dense(oracle, op64, dom, dual)) < 1e-6


@pytest.mark.parametrize("k", [1.0, 3.0, 20.0, 3.0 + 0.6j])
def test_mixed_maxwell_efie_against_fp64_and_oracle(oracle, k):
    """EFIE (RWG domain, SNC dual) under cuda_mixed: moments from the FP32 P1 single-layer core; k = 1, 3, 20
    on a 512-element ellipsoid reach the three phase classes.  Symmetric and per-pair sweeps agree."""
    from cases import oracle_dense

    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    rwg = function_space(grid, "RWG", 0)
    snc = function_space(grid, "SNC", 0)
    a64 = operators.boundary.maxwell.electric_field(rwg, rwg, snc, k).weak_form().tensor
    op = operators.boundary.maxwell.electric_field(rwg, rwg, snc, k, device_interface="cuda_mixed")
    amx = op.weak_form().tensor
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err
    assert rel_fro(amx.cpu().numpy(), oracle_dense(oracle, op, rwg, snc)) < 1e-6
    n = rwg.global_dof_count
    outs = []
    for sym in (True, False):
        a = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
        regular_into(a, op.descriptor, rwg, snc, Parameters(), precision=_lib.MIXED, symmetric=sym)
        singular_into_dense(a, op.descriptor, rwg, snc, Parameters())
        outs.append(a)
    assert (torch.linalg.norm(outs[0] - outs[1]) / torch.linalg.norm(outs[1])).item() < 1e-6
    assert (torch.linalg.norm(outs[0] - a64) / torch.linalg.norm(a64)).item() < 1e-6


@pytest.mark.parametrize("k", [1.0, 3.0, 20.0, 3.0 + 0.6j])
def test_mixed_maxwell_mfie_against_fp64_and_oracle(oracle, k):
    """MFIE (RWG domain, SNC dual) under cuda_mixed: the nine FP32 moments of e^{ikr}(ikr - 1)/r^3 and the
    FP64 determinants det(P_ti - P_sj, J_t^a, J_s^b); k = 1, 3, 20 on a 512-element ellipsoid reach the three
    phase classes.  Symmetric and per-pair sweeps agree."""
    from cases import oracle_dense

    from bempp_cuda import _lib, assembly, operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 1.0)
    rwg = function_space(grid, "RWG", 0)
    snc = function_space(grid, "SNC", 0)
    a64 = operators.boundary.maxwell.magnetic_field(rwg, rwg, snc, k).weak_form().tensor
    op = operators.boundary.maxwell.magnetic_field(rwg, rwg, snc, k, device_interface="cuda_mixed")
    assembly.FP64_FALLBACKS.clear()
    amx = op.weak_form().tensor
    assert not assembly.FP64_FALLBACKS  # the mixed kernel ran
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err
    assert rel_fro(amx.cpu().numpy(), oracle_dense(oracle, op, rwg, snc)) < 1e-6
    n = rwg.global_dof_count
    outs = []
    for sym in (True, False):
        a = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
        regular_into(a, op.descriptor, rwg, snc, Parameters(), precision=_lib.MIXED, symmetric=sym)
        singular_into_dense(a, op.descriptor, rwg, snc, Parameters())
        outs.append(a)
    assert (torch.linalg.norm(outs[0] - outs[1]) / torch.linalg.norm(outs[1])).item() < 1e-6
    assert (torch.linalg.norm(outs[0] - a64) / torch.linalg.norm(a64)).item() < 1e-6


def test_operators_without_mixed_kernel_warn_and_run_fp64():
    """cuda_mixed on an operator without a mixed-precision kernel (a negative real wavenumber on P1: the
    mixed kernels measure lengths in units of 1 / Re k) warns once (MixedPrecisionFallback) and gives the
    FP64 weak form."""
    import warnings

    from bempp_cuda import assembly, operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(2)
    p1 = function_space(grid, "P", 1)
    assembly.FP64_FALLBACKS.clear()
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        mixed = operators.boundary.helmholtz.single_layer(p1, p1, p1, -2.0,
                                                          device_interface="cuda_mixed").weak_form().A
    assert any(issubclass(w.category, assembly.MixedPrecisionFallback) for w in caught)
    fp64 = operators.boundary.helmholtz.single_layer(p1, p1, p1, -2.0).weak_form().A
    assert np.array_equal(mixed, fp64) or np.linalg.norm(mixed - fp64) <= 1e-15 * np.linalg.norm(fp64)


@pytest.mark.parametrize("family,name,k", [("helmholtz", "single_layer", 4.0), ("helmholtz", "double_layer", 4.0),
                                           ("laplace", "adjoint_double_layer", None),
                                           ("modified_helmholtz", "hypersingular", 2.0)])
@pytest.mark.parametrize("kind", ["DP1", "P1 half sphere"])
def test_mixed_p1_other_spaces(oracle, kind, family, name, k):
    """The mixed P1 kernels on DP1 (no shared dofs: each warp's 96 slots are 96 columns) and on a P1 space
    restricted to half the sphere (its boundary vertices carry zero multipliers): within 1e-6 of FP64 and
    the oracle."""
    from cases import oracle_dense

    from bempp_cuda import assembly
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    if kind == "DP1":
        sp = function_space(grid, "DP", 1)
    else:
        cent = grid.vertices[:, grid.elements].mean(axis=1)
        sp = function_space(grid, "P", 1, support_elements=np.flatnonzero(cent[2] > 0.0))
    path = family + "." + name
    a64 = _op(path, sp, k, "cuda").weak_form().tensor
    assembly.FP64_FALLBACKS.clear()
    amx = _op(path, sp, k, "cuda_mixed").weak_form().tensor
    assert not assembly.FP64_FALLBACKS  # a mixed kernel ran
    err = (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item()
    assert 0.0 < err < 1e-6, err
    assert rel_fro(amx.cpu().numpy(), oracle_dense(oracle, _op(path, sp, k, "cuda"), sp, sp)) < 1e-6
