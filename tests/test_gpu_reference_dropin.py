"""User scripts of the real reference, unchanged but for device_interface="cuda" (run on a B200).

The unmodified bempp_cl installed under baseline/_ref (oracle/reference.py;
skipped when it is not installed) builds its own grid, spaces and operators;
``bempp_cuda.plugin.install()`` registers the cuda interface in its
dispatcher.  Each weak form / potential assembled through the reference's
API on the GPU is compared with the same call on the reference's own Numba
path, run live here: 1e-12 relative Frobenius for "cuda", 1e-6 for
"cuda_mixed".  The last test solves a scattering problem with the
reference's own GMRES on both paths.
"""

import numpy as np
import pytest

from oracle import reference

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
bempp_cl = reference.load()


@pytest.fixture(scope="module", autouse=True)
def _setup():
    if bempp_cl is None:
        pytest.skip(str(reference.reason()))
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bempp_cuda import plugin

    plugin.install()


@pytest.fixture(scope="module")
def grid():
    from bempp_cuda.shapes import regular_sphere

    return reference.grid_from(regular_sphere(2))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


CASES = [
    ("laplace.single_layer", ("DP", 0), ("DP", 0), ()),
    ("laplace.hypersingular", ("P", 1), ("P", 1), ()),
    ("helmholtz.single_layer", ("DP", 0), ("DP", 0), (2.5,)),
    ("helmholtz.double_layer", ("P", 1), ("P", 1), (2.5,)),
    ("helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), (2.5 + 1j,)),
    ("helmholtz.hypersingular", ("P", 1), ("P", 1), (2.5,)),
    ("modified_helmholtz.single_layer", ("DP", 0), ("DP", 0), (1.5,)),
    ("maxwell.electric_field", ("RWG", 0), ("SNC", 0), (2.5,)),
    ("maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), (2.5,)),
]


def _factory(root, path):
    obj = root
    for part in path.split("."):
        obj = getattr(obj, part)
    return obj


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_weak_form_cuda_equals_numba(grid, case):
    path, dsp, tsp, args = case
    domain = bempp_cl.api.function_space(grid, *dsp)
    dual = bempp_cl.api.function_space(grid, *tsp)
    f = _factory(bempp_cl.api.operators.boundary, path)
    ref = f(domain, domain, dual, *args, assembler="dense", device_interface="numba").weak_form().A
    got = f(domain, domain, dual, *args, assembler="dense", device_interface="cuda").weak_form().A
    assert got.shape == ref.shape and got.dtype == ref.dtype
    assert _rel(got, ref) < 1e-12, path
    mixed = f(domain, domain, dual, *args, assembler="dense", device_interface="cuda_mixed").weak_form().A
    assert _rel(mixed, ref) < 1e-6, path


@pytest.mark.parametrize("path,kind,args", [
    ("helmholtz.single_layer", ("P", 1), (2.5,)),
    ("helmholtz.double_layer", ("P", 1), (2.5 + 0.5j,)),
    ("laplace.single_layer", ("DP", 0), ()),
    ("maxwell.electric_field", ("RWG", 0), (2.0,)),
])
def test_potential_cuda_equals_numba(grid, path, kind, args):
    space = bempp_cl.api.function_space(grid, *kind)
    rng = np.random.default_rng(7)
    coeffs = rng.standard_normal(space.global_dof_count) + 1j * rng.standard_normal(space.global_dof_count)
    fun = bempp_cl.api.GridFunction(space, coefficients=coeffs)
    pts = rng.standard_normal((3, 64))
    pts *= (1.5 + rng.random(64)) / np.linalg.norm(pts, axis=0)
    f = _factory(bempp_cl.api.operators.potential, path)
    ref = f(space, pts, *args, device_interface="numba").evaluate(fun)
    got = f(space, pts, *args, device_interface="cuda").evaluate(fun)
    assert got.shape == ref.shape
    assert _rel(got, ref) < 1e-12, path


def test_combined_field_solve_through_reference_api(grid):
    """Sound-soft scattering with the reference's own operator algebra, projections and GMRES."""
    k = 3.0
    space = bempp_cl.api.function_space(grid, "DP", 0)
    H = bempp_cl.api.operators.boundary.helmholtz
    ident = bempp_cl.api.operators.boundary.sparse.identity(space, space, space)

    @bempp_cl.api.complex_callable
    def incident(x, n, domain_index, result):
        result[0] = -np.exp(1j * k * x[2])

    rhs = bempp_cl.api.GridFunction(space, fun=incident)
    sols = {}
    for interface in ("numba", "cuda"):
        slp = H.single_layer(space, space, space, k, assembler="dense", device_interface=interface)
        dlp = H.double_layer(space, space, space, k, assembler="dense", device_interface=interface)
        lhs = dlp - 0.5 * ident - 1j * k * slp
        sol, info = bempp_cl.api.linalg.gmres(lhs, rhs, tol=1e-10)
        assert info == 0
        sols[interface] = sol.coefficients
    assert _rel(sols["cuda"], sols["numba"]) < 1e-9
