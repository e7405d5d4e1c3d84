"""Mixed-precision Maxwell far fields and magnetic potential (run on a B200).

``device_interface="cuda_mixed"`` evaluates the magnetic far field with the
phase e^{-i k x . y} split about the element centroids (FP64 per direction
and element, FP32 per source): V = sum kv v, then i k (x x V) per direction
in FP64.  Held to the mixed-precision bound (1e-6 relative Frobenius)
against the oracle and the FP64 path, with k R in each phase class and a
complex wavenumber (whose imaginary part enters the i k factor only, as in
the FP64 kernel).  The electric far field's divergence sum cancels between
neighbouring elements, which FP32 element sums do not survive: it stays
FP64 under cuda_mixed, as does the electric potential.  The magnetic
potential runs mixed: h = (ir' - 1) e^{i theta} / r'^3 times d' x v per pair
in FP32 about the element centroids, FP64 per (point, element) and for the
elements next to a point.
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


@pytest.mark.parametrize("kr", [0.3, 0.8, 3.0, 3.0 + 0.5j])
@pytest.mark.parametrize("name", ["magnetic_field"])
def test_mixed_maxwell_far_fields(oracle, name, kr):
    from cases import oracle_potential

    from bempp_cuda import assembly, operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "RWG", 0)
    rng = np.random.default_rng(19)
    dirs = rng.standard_normal((3, 1500))
    dirs = np.concatenate([dirs / np.linalg.norm(dirs, axis=0), np.eye(3)], axis=1)
    k = kr / device_grid(grid).radius
    f = getattr(operators.far_field.maxwell, name)
    n = space.global_dof_count
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assembly.FP64_FALLBACKS.clear()
    mixed = f(space, dirs, k, device_interface="cuda_mixed")
    got = mixed.evaluate_device(coeffs).cpu().numpy()
    assert not assembly.FP64_FALLBACKS  # the mixed kernel ran
    ref = f(space, dirs, k).evaluate_device(coeffs).cpu().numpy()
    assert got.shape == ref.shape == (3, dirs.shape[1])
    assert 0.0 < rel_fro(got, ref) < 1e-6
    assert rel_fro(got, oracle_potential(oracle, mixed, space, coeffs)) < 1e-6


@pytest.mark.parametrize("path", ["potential.maxwell.electric_field", "far_field.maxwell.electric_field"])
def test_mixed_maxwell_without_mixed_kernel_fall_back_to_fp64(path):
    """The electric potential and far field have no mixed kernel: FP64 under cuda_mixed, with a warning."""
    import warnings

    from bempp_cuda import assembly, operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(2)
    space = function_space(grid, "RWG", 0)
    points, dirs = sphere_shell_points(300, 41)
    if path.startswith("far_field"):
        points = dirs
    f = operators
    for part in path.split("."):
        f = getattr(f, part)
    rng = np.random.default_rng(3)
    c = rng.standard_normal(space.global_dof_count) + 1j * rng.standard_normal(space.global_dof_count)
    assembly.FP64_FALLBACKS.clear()
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        a = f(space, points, 2.0, device_interface="cuda_mixed").evaluate_device(c)
    assert any(issubclass(w.category, assembly.MixedPrecisionFallback) for w in caught)
    b = f(space, points, 2.0).evaluate_device(c)
    assert (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item() < 1e-13


@pytest.mark.parametrize("kr", [0.3, 0.8, 3.0, 3.0 + 0.5j])
def test_mixed_maxwell_magnetic_potential(oracle, kr):
    """Magnetic potential under cuda_mixed at 1500 shell points plus points on element centroids and 1e-3
    above the surface (FP64 branch): within 1e-6 of the oracle and of the FP64 path, k R in each phase
    class and a complex wavenumber."""
    from cases import oracle_potential, sphere_shell_points

    from bempp_cuda import assembly, operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "RWG", 0)
    shell, _ = sphere_shell_points(1500, 43)
    cent = grid.vertices[:, grid.elements].mean(axis=1)
    pick = np.random.default_rng(29).choice(cent.shape[1], 40, replace=False)
    points = np.concatenate([shell, cent[:, pick[:20]], cent[:, pick[20:]] * 1.001], axis=1)
    k = kr / device_grid(grid).radius
    f = operators.potential.maxwell.magnetic_field
    rng = np.random.default_rng(31)
    coeffs = rng.standard_normal(space.global_dof_count) + 1j * rng.standard_normal(space.global_dof_count)
    assembly.FP64_FALLBACKS.clear()
    mixed = f(space, points, k, device_interface="cuda_mixed")
    got = mixed.evaluate_device(coeffs).cpu().numpy()
    assert not assembly.FP64_FALLBACKS  # the mixed kernel ran
    ref = f(space, points, k).evaluate_device(coeffs).cpu().numpy()
    assert got.shape == ref.shape == (3, points.shape[1])
    assert 0.0 < rel_fro(got, ref) < 1e-6
    assert rel_fro(got, oracle_potential(oracle, mixed, space, coeffs)) < 1e-6
