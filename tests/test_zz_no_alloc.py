"""The allocation-free potential entry point against the allocating one.

bemppcuda_evaluate_potential_noalloc exists for callers that only hold the
input and output device buffers handed to them by a host application and
cannot allocate device memory themselves (a plugin inside a solver's memory
pool, an embedding runtime without a CUDA allocation binding).  It keeps its
source table in a fixed array inside the library instead of a caller
workspace.  These tests call both entry points through the C ABI on the same
inputs, twice in a row with different coefficients (the shared array keeps the
previous call's contents), and check that an oversized problem is refused
before any work is launched.  The file name sorts last so a stop-at-first-
failure run has executed every other test before this one.
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


def _args(space, descriptor, points, coefficients):
    from bempp_cuda import _lib
    from bempp_cuda.assembly import kernel_ids, kernel_params, regular_rule
    from bempp_cuda.device import device_grid, device_space, ptr

    kernel, assembly = kernel_ids(descriptor)
    qp, qw = regular_rule(4)
    pts = torch.as_tensor(np.ascontiguousarray(points.T), dtype=torch.float64, device="cuda")
    coeff = torch.as_tensor(np.ascontiguousarray(coefficients), dtype=torch.complex128, device="cuda")
    kdim = 3 if assembly in (_lib.ASM_EFIE, _lib.ASM_MFIE) else 1
    result = torch.full((kdim, points.shape[1]), complex(np.nan, np.nan), dtype=torch.complex128, device="cuda")
    args = _lib.PotentialArgs()
    args.kernel = kernel
    args.assembly = assembly
    args.precision = _lib.FP64
    p = kernel_params(descriptor.options)
    for i in range(4):
        args.params[i] = float(p[i])
    args.grid = device_grid(space.grid).record()
    args.space = device_space(space).record()
    args.nq = len(qw)
    args.quad_points = qp.ctypes.data
    args.quad_weights = qw.ctypes.data
    args.npoints = points.shape[1]
    args.points = ptr(pts)
    args.coefficients = ptr(coeff)
    args.result = ptr(result)
    keep = (pts, coeff, qp, qw)
    return args, result, keep


def _reference_call(args):
    """The allocating entry point with a torch-owned workspace."""
    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream, ptr

    lib = _lib.load()
    need = lib.bemppcuda_potential_workspace_bytes(ctypes.byref(args))
    ws = torch.empty(max(need // 8, 1), dtype=torch.float64, device="cuda")
    args.workspace = ptr(ws)
    args.workspace_bytes = need
    _lib.check(lib.bemppcuda_evaluate_potential(ctypes.byref(args), current_stream()))
    torch.cuda.synchronize()
    return ws


@pytest.mark.parametrize("kind", ["helmholtz", "maxwell"])
def test_noalloc_matches_allocating_entry_point_twice(kind):
    from bempp_cuda import _lib, operators
    from bempp_cuda.device import current_stream
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    lib = _lib.load()
    grid = regular_sphere(3)
    rng = np.random.default_rng(11)
    pts = rng.standard_normal((3, 300))
    pts *= (1.5 + 1.5 * rng.random(300)) / np.linalg.norm(pts, axis=0)
    if kind == "helmholtz":
        space = function_space(grid, "P", 1)
        op = operators.potential.helmholtz.single_layer(space, pts, 4.0 + 0.5j)
    else:
        space = function_space(grid, "RWG", 0)
        op = operators.potential.maxwell.electric_field(space, pts, 3.0)
    for call in range(2):
        dofs = rng.standard_normal(space.global_dof_count) + 1j * rng.standard_normal(space.global_dof_count)
        local = space.map_to_full_grid @ dofs
        args_ref, res_ref, keep_ref = _args(space, op.descriptor, pts, local)
        _reference_call(args_ref)
        args_na, res_na, keep_na = _args(space, op.descriptor, pts, local)
        args_na.workspace = None
        args_na.workspace_bytes = 0
        rc = lib.bemppcuda_evaluate_potential_noalloc(ctypes.byref(args_na), current_stream())
        assert rc == _lib.OK, _lib.last_error()
        torch.cuda.synchronize()
        a = res_na.cpu().numpy()
        b = res_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), "call %d left unwritten outputs" % call
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b), "call %d" % call


def test_noalloc_rejects_oversized_problem():
    from bempp_cuda import _lib, operators
    from bempp_cuda.device import current_stream
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    lib = _lib.load()
    grid = regular_sphere(2)
    space = function_space(grid, "DP", 0)
    pts = np.array([[3.0], [0.0], [0.0]])
    op = operators.potential.laplace.single_layer(space, pts)
    args, res, keep = _args(space, op.descriptor, pts, np.ones(grid.number_of_elements))
    # claim a support far larger than the fixed array can hold; the size check comes first
    args.space.nsupport = _lib.NOALLOC_SCRATCH_DOUBLES // (14 * args.nq) + 1
    rc = lib.bemppcuda_evaluate_potential_noalloc(ctypes.byref(args), current_stream())
    assert rc == _lib.ERR_WORKSPACE
    assert "fixed maximum" in _lib.last_error()
    torch.cuda.synchronize()
    assert torch.isnan(res).all()
