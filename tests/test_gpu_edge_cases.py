"""Edge cases and corrupt inputs (run on a B200).

Empty and tiny problems give the right (possibly empty) results; corrupt
inputs — NaN or degenerate geometry, out-of-range indices, mismatched sizes,
invalid row ranges, out-of-range singular pair tables — return an error status
or are skipped without a GPU fault, and the context stays usable.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _usable():
    torch.cuda.synchronize()
    assert torch.ones(8, device="cuda").sum().item() == 8.0


def _geometry_status(verts, elems):
    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream, ptr

    v = torch.as_tensor(np.asarray(verts, dtype=np.float64), device="cuda")
    e = torch.as_tensor(np.asarray(elems, dtype=np.int32), device="cuda")
    geom = torch.empty((_lib.GEOM_FIELDS, e.shape[0]), dtype=torch.float64, device="cuda")
    rc = _lib.load().bemppcuda_grid_geometry(ptr(v), v.shape[0], ptr(e), e.shape[0], ptr(geom), current_stream())
    return rc, _lib.last_error()


def test_nan_and_degenerate_geometry_are_rejected():
    from bempp_cuda import _lib

    tri = [[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]
    rc, msg = _geometry_status([[0.0, 0.0, np.nan], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]], [[0, 1, 2]])
    assert rc == _lib.ERR_INVALID and "non-finite" in msg
    rc, msg = _geometry_status([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [2.0, 0.0, 0.0]], [[0, 1, 2]])  # collinear
    assert rc == _lib.ERR_INVALID and "degenerate" in msg
    rc, msg = _geometry_status(tri, [[0, 1, -1]])
    assert rc == _lib.ERR_INVALID and "out of range" in msg
    rc, msg = _geometry_status(tri, [[0, 1, 2]])
    assert rc == _lib.OK
    _usable()


def test_mismatched_sizes_and_row_ranges_are_rejected():
    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import regular_into
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(2)
    sp = function_space(grid, "DP", 0)
    n = grid.number_of_elements
    d = operators.boundary.helmholtz.single_layer(sp, sp, sp, 3.0).descriptor
    narrow = torch.empty((n, n - 1), dtype=torch.complex128, device="cuda")
    with pytest.raises(_lib.BemppCudaError) as exc:
        regular_into(narrow, d, sp, sp, Parameters(), overwrite=True)
    assert exc.value.status == _lib.ERR_INVALID
    out = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    for rows in ((0, n + 1), (5, 5), (-1, 3)):
        with pytest.raises(_lib.BemppCudaError) as exc:
            regular_into(out, d, sp, sp, Parameters(), overwrite=True, rows=rows)
        assert exc.value.status == _lib.ERR_INVALID
    # a row range needs the symmetric sweep: the mixed tiles measure lengths in units of 1 / Re k and have
    # none for Re k <= 0 -> rejected, not ignored; complex wavenumbers with Re k > 0 and modified
    # Helmholtz sweep in both precisions -> accepted
    di = operators.boundary.helmholtz.single_layer(sp, sp, sp, -3.0).descriptor
    with pytest.raises(_lib.BemppCudaError) as exc:
        regular_into(out, di, sp, sp, Parameters(), precision=_lib.MIXED, overwrite=True, rows=(0, 8))
    assert exc.value.status == _lib.ERR_INVALID
    dm = operators.boundary.modified_helmholtz.single_layer(sp, sp, sp, 2.0).descriptor
    real_out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    regular_into(real_out, dm, sp, sp, Parameters(), precision=_lib.MIXED, overwrite=True, rows=(0, 8))
    dc = operators.boundary.helmholtz.single_layer(sp, sp, sp, 3.0 + 0.5j).descriptor
    regular_into(out, dc, sp, sp, Parameters(), precision=_lib.MIXED, overwrite=True, rows=(0, 8))
    regular_into(out, dc, sp, sp, Parameters(), overwrite=True, rows=(0, 8))
    _usable()


def test_out_of_range_singular_pairs_are_skipped():
    """A caller table with a bad element id or offset: that pair is skipped, the others are assembled."""
    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import singular_into_dense
    from bempp_cuda.device import device_singular_rule
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(1)
    sp = function_space(grid, "DP", 0)
    n = grid.number_of_elements
    d = operators.boundary.laplace.single_layer(sp, sp, sp).descriptor
    ref = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    singular_into_dense(ref, d, sp, sp, Parameters())
    rule = device_singular_rule(grid, 4, sp.support, sp.support)
    saved = (rule.test_elements.clone(), rule.test_offsets.clone())
    try:
        rule.test_elements[0] = n + 1000  # element id past the grid
        rule.test_offsets[1] = rule.npoints_table  # point range past the table
        out = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        singular_into_dense(out, d, sp, sp, Parameters())
        _usable()
    finally:
        rule.test_elements.copy_(saved[0])
        rule.test_offsets.copy_(saved[1])
    diff = (out - ref).abs() > 1e-15 * ref.abs().max()
    assert int(diff.sum().item()) <= 2  # only the two corrupted pairs are missing


def test_empty_and_tiny_problems():
    from bempp_cuda import operators
    from bempp_cuda.grid import Grid
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    # one triangle: a 1 x 1 DP0 matrix (the coincident pair only) against the oracle
    from oracle import oracle as orc
    from bempp_cuda.quadrature import SingularPairs, triangle_rule

    g1 = Grid(np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, 0.0]]), np.array([[0], [1], [2]], dtype=np.uint32))
    sp1 = function_space(g1, "DP", 0)
    for k in (None, 2.0):
        op = (operators.boundary.laplace.single_layer(sp1, sp1, sp1) if k is None
              else operators.boundary.helmholtz.single_layer(sp1, sp1, sp1, k))
        a = op.weak_form().tensor.cpu().numpy()
        qp, qw = triangle_rule(4)
        rule = SingularPairs(g1, 4, sp1.support, sp1.support).arrays()
        dsc = op.descriptor
        b = orc.assemble_dense(dsc.kernel_type, dsc.assembly_type, dsc.options, dsc.is_complex, sp1, sp1, qp, qw, rule)
        assert a.shape == (1, 1) and abs(a[0, 0] - b[0, 0]) <= 1e-13 * abs(b[0, 0])
    # octahedron (8 elements): every symmetric tile is a diagonal tile
    g0 = regular_sphere(0)
    sp0 = function_space(g0, "DP", 0)
    for sym in (True, False):
        from bempp_cuda.assembly import regular_into
        from bempp_cuda.operators import Parameters

        out = torch.full((8, 8), np.nan, dtype=torch.complex128, device="cuda")
        d = operators.boundary.helmholtz.double_layer(sp0, sp0, sp0, 1.5).descriptor
        regular_into(out, d, sp0, sp0, Parameters(), overwrite=True, symmetric=sym)
        assert torch.isfinite(torch.view_as_real(out)).all()
    # potentials at zero points and an empty support
    pot = operators.potential.laplace.single_layer(sp0, np.zeros((3, 0)))
    assert pot.evaluate(np.ones(8)).shape == (1, 0)
    empty = function_space(g0, "DP", 0, support_elements=np.arange(0))
    assert empty.global_dof_count == 0
    _usable()


def test_batch_of_one_and_empty_batch():
    from bempp_cuda import _lib
    from bempp_cuda.batch import BatchAssembler
    from bempp_cuda.shapes import regular_sphere

    g = regular_sphere(2)
    ba = BatchAssembler([g], [4.0])
    ba.launch()
    torch.cuda.synchronize()
    assert torch.isfinite(torch.view_as_real(ba.outputs[0])).all()
    with pytest.raises(ValueError):
        BatchAssembler([], [])
    ba.args.nproblems = 0
    rc = _lib.load().bemppcuda_batch_launch(ctypes.byref(ba.args), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _lib.ERR_INVALID
    _usable()


def test_shape_gradient_on_the_octahedron():
    """The smallest closed grid: every pair is adjacent except the opposite faces."""
    from bempp_cuda.shape_gradient import FarFieldObjective, fibonacci_directions
    from bempp_cuda.shapes import regular_sphere

    obj = FarFieldObjective(regular_sphere(0), directions=fibonacci_directions(8))
    x0 = obj.vertices.clone()
    value, state = obj.evaluate(x0, 2.0, keep=True)
    vgrad, kgrad = obj.gradient(state, 2.0)
    h = 1e-6
    for v, c in ((0, 0), (3, 2), (5, 1)):
        xp = x0.clone()
        xm = x0.clone()
        xp[v, c] += h
        xm[v, c] -= h
        fd = (obj.evaluate(xp, 2.0).item() - obj.evaluate(xm, 2.0).item()) / (2 * h)
        assert abs(vgrad[v, c].item() - fd) <= 1e-6 * vgrad.abs().max().item()


def _two_element_grid():
    from bempp_cuda.grid import Grid

    verts = np.array([[0.0, 1.0, 0.0, 1.0], [0.0, 0.0, 1.0, 1.0], [0.0, 0.0, 0.0, 0.2]])
    elems = np.array([[0, 1], [1, 3], [2, 2]], dtype=np.uint32)  # triangles (0,1,2) and (1,3,2) share an edge
    return Grid(verts, elems)


@pytest.mark.parametrize("which", ["octahedron", "two_elements"])
def test_every_boundary_operator_on_extreme_adjacency(which, oracle):
    """All operator x space cases where (almost) every element pair is adjacent: against the oracle."""
    from cases import BOUNDARY, boundary_operator, oracle_dense

    from bempp_cuda.shapes import regular_sphere

    grid = regular_sphere(0) if which == "octahedron" else _two_element_grid()
    for key in BOUNDARY:
        if which == "two_elements" and key.startswith("maxwell"):
            continue  # one interior edge: RWG / SNC have a single dof; covered on the octahedron
        op, domain, dual = boundary_operator(key, grid)
        got = op.weak_form().tensor.cpu().numpy()
        if domain.global_dof_count == 0 or dual.global_dof_count == 0:
            # P1 on the open two-element grid: every vertex is a boundary vertex, no dofs
            assert got.shape == (dual.global_dof_count, domain.global_dof_count), key
            continue
        ref = oracle_dense(oracle, op, domain, dual)
        scale = max(np.linalg.norm(ref), 1e-300)
        assert np.linalg.norm(got - ref) <= 1e-12 * scale, key


def _open_sphere(level, removed):
    """regular_sphere(level) without its last ``removed`` elements: an open surface with boundary edges."""
    from bempp_cuda.grid import Grid
    from bempp_cuda.shapes import regular_sphere

    g = regular_sphere(level)
    keep = np.arange(g.number_of_elements - removed)
    used = np.unique(g.elements[:, keep])
    remap = -np.ones(g.vertices.shape[1], dtype=np.int64)
    remap[used] = np.arange(len(used))
    return Grid(g.vertices[:, used], remap[g.elements[:, keep]].astype(np.uint32))


@pytest.mark.parametrize("key", ["maxwell_efie_rwg_snc", "maxwell_mfie_rwg_snc", "helmholtz_slp_p1_p1",
                                 "helmholtz_hyp_p1_p1", "helmholtz_dlp_p1_p1"])
def test_specialised_kernels_on_an_open_surface(oracle, key):
    """Boundary edges / vertices carry no dof (zero multipliers): the RWG and P1 kernels skip them."""
    from cases import BOUNDARY, boundary_operator, oracle_dense

    if key not in BOUNDARY:
        pytest.skip("case not defined")
    grid = _open_sphere(3, 37)
    op, domain, dual = boundary_operator(key, grid)
    got = op.weak_form().tensor.cpu().numpy()
    ref = oracle_dense(oracle, op, domain, dual)
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), key


def test_mixed_p1_on_an_open_surface():
    from bempp_cuda import operators
    from bempp_cuda.space import function_space

    sp = function_space(_open_sphere(3, 37), "P", 1)
    for name in ("single_layer", "hypersingular"):
        f = getattr(operators.boundary.helmholtz, name)
        a64 = f(sp, sp, sp, 4.0).weak_form().tensor
        amx = f(sp, sp, sp, 4.0, device_interface="cuda_mixed").weak_form().tensor
        assert (torch.linalg.norm(amx - a64) / torch.linalg.norm(a64)).item() < 1e-6, name
