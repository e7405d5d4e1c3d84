"""The drop-in boundary against the real reference package (CPU).

Uses the unmodified bempp_cl installed under baseline/_ref (oracle/reference.py);
skipped when it is not installed.  Checks that the reference's own grids,
function spaces and operator descriptors produce exactly the inputs the cuda
device interface uploads from this package's objects, and that after
``plugin.install()`` the reference's dispatcher (core/dispatcher.py:4-55)
still routes "numba" to its own assemblers while "cuda" reaches this package,
which fails loudly without a GPU instead of falling back to the CPU.
"""

import numpy as np
import pytest

from oracle import reference

bempp_cl = reference.load()
pytestmark = pytest.mark.skipif(bempp_cl is None, reason=str(reference.reason()))

SPACES = [("DP", 0), ("P", 1), ("DP", 1), ("RWG", 0), ("SNC", 0)]


def _columns(a):
    a = np.asarray(a)
    return sorted(map(tuple, a.T.tolist()))


@pytest.fixture(scope="module")
def grids():
    from bempp_cuda.shapes import regular_sphere

    ours = regular_sphere(2)
    return ours, reference.grid_from(ours)


def test_grid_arrays_and_adjacency(grids):
    from bempp_cuda.device import host_grid_arrays

    ours, ref = grids
    for a, b in zip(host_grid_arrays(ours), host_grid_arrays(ref)):
        assert a.dtype == b.dtype and np.array_equal(a, b)
    # the same element pairs with the same local vertex indices; the column order follows each
    # package's sparse adjacency walk, and the pair order does not enter the assembled matrix
    assert _columns(ours.edge_adjacency) == _columns(ref.edge_adjacency)
    assert _columns(ours.vertex_adjacency) == _columns(ref.vertex_adjacency)
    np.testing.assert_allclose(ours.volumes, ref.volumes, rtol=1e-15)
    np.testing.assert_allclose(ours.normals, ref.normals, rtol=0, atol=1e-15)


@pytest.mark.parametrize("kind", SPACES)
def test_space_arrays_equal(grids, kind):
    from bempp_cuda.device import host_space_arrays
    from bempp_cuda.space import function_space

    ours, ref = grids
    a = host_space_arrays(function_space(ours, *kind))
    b = host_space_arrays(bempp_cl.api.function_space(ref, *kind))
    assert a.keys() == b.keys()
    for name in a:
        assert np.array_equal(np.asarray(a[name]), np.asarray(b[name])), (kind, name)


@pytest.mark.parametrize("kind", SPACES)
def test_singular_pairs_from_reference_objects(grids, kind):
    from bempp_cuda.quadrature import SingularPairs
    from bempp_cuda.space import function_space

    ours, ref = grids
    sp_o = function_space(ours, *kind).localised_space
    sp_r = bempp_cl.api.function_space(ref, *kind).localised_space
    a = SingularPairs(ours, 4, sp_o.support, sp_o.support).arrays()
    b = SingularPairs(ref, 4, sp_r.support, sp_r.support).arrays()
    for x, y in zip(a[:3], b[:3]):  # point tables and weights
        assert x.dtype == y.dtype and np.array_equal(x, y)
    # per pair: test / trial element, the three table offsets and the point count
    assert _columns(np.vstack(a[3:])) == _columns(np.vstack(b[3:]))


def test_reference_descriptors_map_to_kernels(grids):
    """Every reference boundary operator of the path names a kernel / assembly the library knows, with
    the same descriptor fields as this package's factories (the reference keeps potential descriptors
    inside its assembler; the GPU drop-in test evaluates those potentials end to end)."""
    from bempp_cuda import operators
    from bempp_cuda.assembly import kernel_ids, kernel_params
    from bempp_cuda.space import function_space

    ours, ref = grids
    ops = bempp_cl.api.operators.boundary
    sp_r = bempp_cl.api.function_space(ref, "P", 1)
    rwg, snc = bempp_cl.api.function_space(ref, "RWG", 0), bempp_cl.api.function_space(ref, "SNC", 0)
    sp_o = function_space(ours, "P", 1)
    rwg_o, snc_o = function_space(ours, "RWG", 0), function_space(ours, "SNC", 0)
    theirs = [
        ops.laplace.single_layer(sp_r, sp_r, sp_r, assembler="dense"),
        ops.laplace.hypersingular(sp_r, sp_r, sp_r, assembler="dense"),
        ops.helmholtz.double_layer(sp_r, sp_r, sp_r, 2.5, assembler="dense"),
        ops.helmholtz.hypersingular(sp_r, sp_r, sp_r, 2.5 + 1j, assembler="dense"),
        ops.modified_helmholtz.adjoint_double_layer(sp_r, sp_r, sp_r, 1.5, assembler="dense"),
        ops.maxwell.electric_field(rwg, rwg, snc, 2.0, assembler="dense"),
        ops.maxwell.magnetic_field(rwg, rwg, snc, 2.0, assembler="dense"),
    ]
    mine = [
        operators.boundary.laplace.single_layer(sp_o, sp_o, sp_o),
        operators.boundary.laplace.hypersingular(sp_o, sp_o, sp_o),
        operators.boundary.helmholtz.double_layer(sp_o, sp_o, sp_o, 2.5),
        operators.boundary.helmholtz.hypersingular(sp_o, sp_o, sp_o, 2.5 + 1j),
        operators.boundary.modified_helmholtz.adjoint_double_layer(sp_o, sp_o, sp_o, 1.5),
        operators.boundary.maxwell.electric_field(rwg_o, rwg_o, snc_o, 2.0),
        operators.boundary.maxwell.magnetic_field(rwg_o, rwg_o, snc_o, 2.0),
    ]
    for r, m in zip(theirs, mine):
        dr, dm = r.descriptor, m.descriptor
        assert kernel_ids(dr) == kernel_ids(dm)
        assert (dr.identifier, dr.kernel_type, dr.assembly_type, dr.is_complex) == (
            dm.identifier, dm.kernel_type, dm.assembly_type, dm.is_complex)
        assert np.array_equal(kernel_params(dr.options), kernel_params(dm.options))


def test_plugin_keeps_numba_and_routes_cuda(grids):
    """After install(): "numba" still assembles through the reference's own Numba path (equal to the
    oracle), "cuda" reaches this package (no CUDA device here: a RuntimeError, no CPU fallback),
    and an unknown interface still raises the reference's ValueError."""
    import torch

    from bempp_cuda import plugin
    from bempp_cuda.quadrature import SingularPairs, triangle_rule
    from oracle import oracle as orc

    _, ref = grids
    plugin.install()
    sp = bempp_cl.api.function_space(ref, "DP", 0)
    slp = bempp_cl.api.operators.boundary.helmholtz.single_layer
    op = slp(sp, sp, sp, 2.5, assembler="dense", device_interface="numba")
    mat = op.weak_form().A
    d = op.descriptor
    qp, qw = triangle_rule(4)
    rule = SingularPairs(ref, 4, sp.support, sp.support).arrays()
    expect = orc.assemble_dense(d.kernel_type, d.assembly_type, d.options, True, sp, sp, qp, qw, rule)
    assert np.linalg.norm(mat - expect) / np.linalg.norm(expect) < 1e-12
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError, match="CUDA device"):
            slp(sp, sp, sp, 2.5, assembler="dense", device_interface="cuda").weak_form()
    with pytest.raises(ValueError):
        slp(sp, sp, sp, 2.5, assembler="dense", device_interface="vulkan").weak_form()
