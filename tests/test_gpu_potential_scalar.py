"""The per-point scalar potential kernel against the oracle (run on a B200).

Laplace, Helmholtz (real and complex wavenumber) and modified Helmholtz
single / double layer potentials go through ``potential_scalar``: a thread per evaluation point, sources staged in
shared memory, the support split into chunks added with atomics, and the
Helmholtz phase factored about each element's centroid when k R <= 1
(R = largest centroid-to-vertex distance).  The cases below reach every phase
class (k R <= 1/2, <= 1, above 1, and R unknown), both rule branches (six
points and a general rule size), a single chunk (direct store) and many
chunks, ragged point counts, and points on element centroids and very close to
the surface.  Tolerance: 1e-12 relative Frobenius norm, as for the other FP64
paths.
"""

import ctypes

import numpy as np
import pytest

from conftest import rel_fro

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _operator(name, space, points, k, parameters=None):
    from bempp_cuda import operators

    family = operators.potential.laplace if k is None else operators.potential.helmholtz
    factory = getattr(family, name)
    return factory(space, points, parameters=parameters) if k is None else factory(space, points, k,
                                                                                   parameters=parameters)


def _check(oracle, op, space, seed=5, tol=1e-12):
    from cases import oracle_potential

    rng = np.random.default_rng(seed)
    n = space.global_dof_count
    coeffs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    got = op.evaluate_device(coeffs).cpu().numpy()
    ref = oracle_potential(oracle, op, space, coeffs)
    assert got.shape == ref.shape
    assert np.all(np.isfinite(got))
    assert rel_fro(got, ref) < tol
    return got


@pytest.mark.parametrize("kr", [0.3, 0.8, 3.0])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("family", ["DP0", "P1"])
def test_helmholtz_every_phase_class(oracle, kr, name, family):
    """k R = 0.3, 0.8, 3.0 select the three phase classes; 3000 shell points split into several chunks."""
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "DP", 0) if family == "DP0" else function_space(grid, "P", 1)
    k = kr / device_grid(grid).radius
    points, _ = sphere_shell_points(3000, 17)
    _check(oracle, _operator(name, space, points, k), space)


@pytest.mark.parametrize("k", [2.5 + 1.0j, 6.0 + 0.3j])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
def test_helmholtz_complex_wavenumber(oracle, k, name):
    """Complex wavenumbers (phase class 3: exp(-Im k r) per point-source pair, no centroid factoring)."""
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "P", 1)
    points, _ = sphere_shell_points(2000, 19)
    _check(oracle, _operator(name, space, points, k), space)


@pytest.mark.parametrize("omega", [0.7, 4.0])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("family", ["DP0", "P1"])
def test_modified_helmholtz(oracle, omega, name, family):
    """Modified Helmholtz potentials: the Laplace kernels times exp(-w r) (single) or exp(-w r) (1 + w r)."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "DP", 0) if family == "DP0" else function_space(grid, "P", 1)
    points, _ = sphere_shell_points(1500, 23)
    op = getattr(operators.potential.modified_helmholtz, name)(space, points, omega)
    _check(oracle, op, space)


@pytest.mark.parametrize("kr", [None, 0.3, 0.8, 3.0])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("family", ["DP0", "P1"])
def test_mixed_precision_potentials(oracle, kr, name, family):
    """``device_interface="cuda_mixed"``: FP32 point-source pairs (Laplace, and Helmholtz in each phase
    class) within 1e-6 of the oracle and different from the FP64 path."""
    from bempp_cuda import operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "DP", 0) if family == "DP0" else function_space(grid, "P", 1)
    points, _ = sphere_shell_points(3000, 29)
    if kr is None:
        family_ops, args = operators.potential.laplace, ()
    else:
        family_ops, args = operators.potential.helmholtz, (kr / device_grid(grid).radius,)
    mixed = getattr(family_ops, name)(space, points, *args, device_interface="cuda_mixed")
    fp64 = getattr(family_ops, name)(space, points, *args)
    got = _check(oracle, mixed, space, tol=1e-6)
    ref = _check(oracle, fp64, space)
    assert 0.0 < rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("k", [0.3 + 0.1j, 0.8 + 0.4j, 3.0 + 0.5j, 6.0 + 3.0j, "w1.5", "w12"])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("family", ["DP0", "P1"])
def test_mixed_potentials_complex_and_modified(oracle, family, name, k):
    """cuda_mixed for complex wavenumbers (Re k R in each phase class, Im k up to Re k / 2) and modified
    Helmholtz (w = 1.5, 12): FP32 point-source pairs with the amplitude e^{-beta r'} split about the element
    centroids, within 1e-6 of the oracle and of the FP64 path; points on centroids and 1e-3 above the
    surface take the FP64 branch."""
    from bempp_cuda import assembly, operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "DP", 0) if family == "DP0" else function_space(grid, "P", 1)
    shell, _ = sphere_shell_points(1500, 37)
    cent = grid.vertices[:, grid.elements].mean(axis=1)
    pick = np.random.default_rng(13).choice(cent.shape[1], 40, replace=False)
    points = np.concatenate([shell, cent[:, pick[:20]], cent[:, pick[20:]] * 1.001], axis=1)
    if isinstance(k, str):
        fam, args = operators.potential.modified_helmholtz, (float(k[1:]),)
    else:
        fam, args = operators.potential.helmholtz, (k.real / device_grid(grid).radius + 1j * k.imag / device_grid(grid).radius,)
    assembly.FP64_FALLBACKS.clear()
    mixed = getattr(fam, name)(space, points, *args, device_interface="cuda_mixed")
    got = _check(oracle, mixed, space, tol=1e-6)
    assert not assembly.FP64_FALLBACKS  # the mixed kernel ran
    ref = _check(oracle, getattr(fam, name)(space, points, *args), space)
    assert 0.0 < rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
def test_laplace_points_near_the_surface(oracle, name):
    """Points on element centroids, 1e-3 above the surface and far away, with a ragged count (257)."""
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "P", 1)
    v = grid.vertices
    e = grid.elements
    cent = v[:, e].mean(axis=1)  # (3, ne) element centroids
    rng = np.random.default_rng(3)
    pick = rng.choice(cent.shape[1], 100, replace=False)
    near = cent[:, pick[:50]] * 1.001
    far = rng.standard_normal((3, 157)) * 5.0
    points = np.concatenate([cent[:, pick[50:]], near, far], axis=1)
    assert points.shape[1] == 257
    _check(oracle, _operator(name, space, points, None), space)
    _check(oracle, _operator(name, space, points, 4.0), space)


@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("k", [None, 4.0])
def test_mixed_points_near_the_surface(oracle, name, k):
    """cuda_mixed with points on element centroids and 1e-3 above the surface: the elements next to a point
    are evaluated in FP64 (the FP32 offsets would cancel there), so the result stays within 1e-6."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "P", 1)
    cent = grid.vertices[:, grid.elements].mean(axis=1)
    rng = np.random.default_rng(11)
    pick = rng.choice(cent.shape[1], 100, replace=False)
    points = np.concatenate([cent[:, pick[:50]], cent[:, pick[50:]] * 1.001, rng.standard_normal((3, 57)) * 5.0],
                            axis=1)
    family, args = (operators.potential.laplace, ()) if k is None else (operators.potential.helmholtz, (k,))
    mixed = getattr(family, name)(space, points, *args, device_interface="cuda_mixed")
    _check(oracle, mixed, space, tol=1e-6)


@pytest.mark.parametrize("order", [2, 6])
def test_general_rule_size(oracle, order):
    """Rules with other than six points take the runtime-size branch of the kernel."""
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(2)
    space = function_space(grid, "P", 1)
    prm = Parameters()
    prm.quadrature.regular = order
    points, _ = sphere_shell_points(700, 9)
    for name in ("single_layer", "double_layer"):
        for k in (None, 3.0):
            _check(oracle, _operator(name, space, points, k, parameters=prm), space)
    # the mixed kernel with the same rule sizes
    from bempp_cuda import operators

    for k in (None, 3.0):
        family, args = (operators.potential.laplace, ()) if k is None else (operators.potential.helmholtz, (k,))
        op = family.double_layer(space, points, *args, parameters=prm, device_interface="cuda_mixed")
        _check(oracle, op, space, tol=1e-6)


def test_single_chunk_and_single_point(oracle):
    """The octahedron (8 elements) is one chunk: the kernel stores instead of adding atomically."""
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(0)
    space = function_space(grid, "DP", 0)
    for points in (np.array([[2.0], [0.5], [-0.3]]), np.random.default_rng(1).standard_normal((3, 600)) * 3.0):
        for k in (None, 1.5):
            for name in ("single_layer", "double_layer"):
                _check(oracle, _operator(name, space, points, k), space)


def test_unknown_phase_radius_matches_factored_result():
    """A caller that leaves phase_radius at 0 gets the unfactored phase; both agree to FP64 accuracy."""
    from bempp_cuda import _lib
    from bempp_cuda.assembly import kernel_ids, potential_workspace_bytes, regular_rule
    from bempp_cuda.device import current_stream, device_grid, device_space, ptr
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(3)
    space = function_space(grid, "P", 1)
    points, _ = sphere_shell_points(1000, 2)
    pts = torch.as_tensor(np.ascontiguousarray(points.T), device="cuda")
    rng = np.random.default_rng(4)
    local = space.map_to_full_grid @ (rng.standard_normal(space.global_dof_count) + 0j)
    coeff = torch.as_tensor(np.ascontiguousarray(local, dtype=np.complex128), device="cuda")
    op = _operator("single_layer", space, points, 5.0)
    kernel, assembly = kernel_ids(op.descriptor)
    qp, qw = regular_rule(4)
    results = []
    for radius in (0.0, 1.0001 * device_grid(grid).radius):
        out = torch.full((1, points.shape[1]), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
        args = _lib.PotentialArgs()
        args.kernel = kernel
        args.assembly = assembly
        args.precision = _lib.FP64
        args.params[0] = 5.0
        args.grid = device_grid(grid).record()
        args.space = device_space(space).record()
        args.nq = len(qw)
        args.quad_points = qp.ctypes.data
        args.quad_weights = qw.ctypes.data
        args.npoints = points.shape[1]
        args.points = ptr(pts)
        args.coefficients = ptr(coeff)
        args.result = ptr(out)
        need = potential_workspace_bytes(args)
        ws = torch.empty(need // 8, dtype=torch.float64, device="cuda")
        args.workspace = ptr(ws)
        args.workspace_bytes = need
        args.phase_radius = radius
        _lib.check(_lib.load().bemppcuda_evaluate_potential(ctypes.byref(args), current_stream()))
        torch.cuda.synchronize()
        results.append(out.cpu().numpy())
    assert np.all(np.isfinite(results[0]))
    assert rel_fro(results[1], results[0]) < 1e-13


def test_mixed_precision_argument_checks():
    """Through the C ABI: an unknown precision is invalid; MIXED for a Maxwell potential is unsupported
    (the host layer then evaluates in FP64); MIXED needs the grid's phase radius (it bounds the points
    that take FP64 sources next to the surface) and refuses an unknown one."""
    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import kernel_ids, potential_workspace_bytes, regular_rule
    from bempp_cuda.device import current_stream, device_grid, device_space, ptr
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space
    from cases import sphere_shell_points

    grid = regular_sphere(2)
    points, _ = sphere_shell_points(300, 5)
    pts = torch.as_tensor(np.ascontiguousarray(points.T), device="cuda")
    qp, qw = regular_rule(4)

    def args_for(space, op, k):
        kernel, assembly = kernel_ids(op.descriptor)
        nshape = space.number_of_shape_functions
        coeff = torch.ones(grid.number_of_elements * nshape, dtype=torch.complex128, device="cuda")
        kdim = 3 if assembly != _lib.ASM_SCALAR else 1
        out = torch.zeros((kdim, points.shape[1]), dtype=torch.complex128, device="cuda")
        a = _lib.PotentialArgs()
        a.kernel, a.assembly = kernel, assembly
        a.params[0] = k
        a.grid = device_grid(grid).record()
        a.space = device_space(space).record()
        a.nq = len(qw)
        a.quad_points, a.quad_weights = qp.ctypes.data, qw.ctypes.data
        a.npoints = points.shape[1]
        a.points, a.coefficients, a.result = ptr(pts), ptr(coeff), ptr(out)
        need = potential_workspace_bytes(a)
        ws = torch.empty(max(need // 8, 1), dtype=torch.float64, device="cuda")
        a.workspace, a.workspace_bytes = ptr(ws), need
        return a, (coeff, out, ws)

    lib = _lib.load()
    p1 = function_space(grid, "P", 1)
    a, keep = args_for(p1, operators.potential.helmholtz.single_layer(p1, points, 4.0), 4.0)
    a.precision = 7
    assert lib.bemppcuda_evaluate_potential(ctypes.byref(a), current_stream()) == _lib.ERR_INVALID
    a.precision = _lib.MIXED
    a.phase_radius = 0.0  # unknown: the near-surface FP64 treatment has no bound, so MIXED refuses it
    assert lib.bemppcuda_evaluate_potential(ctypes.byref(a), current_stream()) == _lib.ERR_INVALID
    assert "phase_radius" in _lib.last_error()
    a.phase_radius = 1.0001 * device_grid(grid).radius
    assert lib.bemppcuda_evaluate_potential(ctypes.byref(a), current_stream()) == _lib.OK
    a.precision = _lib.FP64
    b, keep_b = args_for(p1, operators.potential.helmholtz.single_layer(p1, points, 4.0), 4.0)
    assert lib.bemppcuda_evaluate_potential(ctypes.byref(b), current_stream()) == _lib.OK
    torch.cuda.synchronize()
    assert rel_fro(keep[1].cpu().numpy(), keep_b[1].cpu().numpy()) < 1e-6
    rwg = function_space(grid, "RWG", 0)
    m, keep_m = args_for(rwg, operators.potential.maxwell.electric_field(rwg, points, 2.0), 2.0)
    m.precision = _lib.MIXED
    assert lib.bemppcuda_evaluate_potential(ctypes.byref(m), current_stream()) == _lib.ERR_UNSUPPORTED
    assert "mixed-precision potentials" in _lib.last_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("kr", [0.3, 0.8, 3.0])
@pytest.mark.parametrize("name", ["single_layer", "double_layer"])
@pytest.mark.parametrize("family", ["DP0", "P1"])
def test_mixed_far_fields(oracle, family, name, kr):
    """cuda_mixed Helmholtz far fields: e^{-i k x . y} split about the element centroids (FP64 phase per
    direction and element, FP32 offsets per source) within 1e-6 of the oracle and of the FP64 path, k R in
    each phase class, 2000 random directions plus the coordinate axes."""
    from bempp_cuda import assembly, operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "DP", 0) if family == "DP0" else function_space(grid, "P", 1)
    rng = np.random.default_rng(17)
    dirs = rng.standard_normal((3, 2000))
    dirs = np.concatenate([dirs / np.linalg.norm(dirs, axis=0), np.eye(3), -np.eye(3)], axis=1)
    k = kr / device_grid(grid).radius
    f = getattr(operators.far_field.helmholtz, name)
    assembly.FP64_FALLBACKS.clear()
    got = _check(oracle, f(space, dirs, k, device_interface="cuda_mixed"), space, tol=1e-6)
    assert not assembly.FP64_FALLBACKS  # the mixed kernel ran
    ref = _check(oracle, f(space, dirs, k), space)
    assert 0.0 < rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("scale", [3.0, 0.5])
def test_mixed_far_field_non_unit_directions(oracle, scale):
    """Directions scaled away from unit length: the mixed far field leaves the phase-class polynomials
    (whose range assumes |x| <= 1) for the reduced ones and stays within 1e-6 of the oracle and FP64."""
    from bempp_cuda import operators
    from bempp_cuda.device import device_grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    space = function_space(grid, "P", 1)
    rng = np.random.default_rng(23)
    dirs = rng.standard_normal((3, 700))
    dirs = scale * dirs / np.linalg.norm(dirs, axis=0)
    k = 0.4 / device_grid(grid).radius  # k R = 0.4: the short polynomials for unit directions
    f = operators.far_field.helmholtz.double_layer
    got = _check(oracle, f(space, dirs, k, device_interface="cuda_mixed"), space, tol=1e-6)
    ref = _check(oracle, f(space, dirs, k), space)
    assert rel_fro(got, ref) < 1e-6


@pytest.mark.parametrize("kind", [("P", 1), ("DP", 0), ("DP", 1), ("RWG", 0)])
def test_device_coefficient_map_equals_sparse_map(kind):
    """The operator's device gather of element-local coefficients (dof index times multiplier per slot,
    zero outside the support) equals ``space.map_to_full_grid @ x`` bit for bit, for full and
    restricted supports, host and device coefficient inputs."""
    from bempp_cuda import operators
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(3)
    # the full grid, and the elements of the upper half (centroid z > 0)
    vertices, elements = np.asarray(grid.vertices), np.asarray(grid.elements)
    upper = np.flatnonzero(vertices[2][elements].mean(axis=0) > 0.0)
    spaces = [function_space(grid, *kind), function_space(grid, *kind, support_elements=upper)]
    rng = np.random.default_rng(11)
    for sp in spaces:
        pot = operators.potential.helmholtz.single_layer(sp, rng.standard_normal((3, 5)) * 3.0, 2.0)
        c = rng.standard_normal(sp.global_dof_count) + 1j * rng.standard_normal(sp.global_dof_count)
        idx, mlt = pot._device_map()
        for coeff in (torch.as_tensor(c, device="cuda"), torch.as_tensor(c)):
            got = coeff.to("cuda").index_select(0, idx) * mlt
            assert np.array_equal(got.cpu().numpy(), sp.map_to_full_grid @ c)
