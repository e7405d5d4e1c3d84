"""Device projections of callables (csrc/project.cu) (run on a B200).

Against the host restatement of the reference's vectorized projection
(tests/shape_oracle.project_callable) for DP0, P1 and DP1 spaces, host and
device callables (<=1e-13 relative), and against the unmodified reference's
own GridFunction.projections (baseline/_ref, when installed; <=1e-12).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


K = 4.0


def host_fun(x, n, domain_index, result):
    result[0] = np.exp(1j * K * x[2]) * (1.0 + 0.5 * n[0]) + x[0] * x[1]


def _device_fun():
    from bempp_cuda.grid_function import device_callable

    @device_callable
    def fun(x, n, domain_index):
        return torch.exp(1j * K * x[2]) * (1.0 + 0.5 * n[0]) + x[0] * x[1]

    return fun


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("kind", [("DP", 0), ("P", 1), ("DP", 1)])
def test_device_projection_matches_host_restatement(kind):
    from shape_oracle import project_callable

    from bempp_cuda.grid_function import GridFunction, project_callable_device
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    sp = function_space(ellipsoid(3, 1.2, 0.9, 0.7), *kind)
    ref = project_callable(host_fun, sp, 4, True)
    got_host_fun = project_callable_device(host_fun, sp).cpu().numpy()
    got_dev_fun = project_callable_device(_device_fun(), sp).cpu().numpy()
    assert _rel(got_host_fun, ref) < 1e-13
    assert _rel(got_dev_fun, ref) < 1e-13
    assert _rel(GridFunction(sp, fun=_device_fun()).projections(sp), ref) < 1e-13


def test_projection_matches_reference_gridfunction():
    from oracle import reference

    bempp_cl = reference.load()
    if bempp_cl is None:
        pytest.skip(str(reference.reason()))
    from bempp_cuda.grid_function import project_callable_device
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    ours = regular_sphere(2)
    ref_grid = reference.grid_from(ours)

    @bempp_cl.api.complex_callable
    def fun(x, n, domain_index, result):
        result[0] = np.exp(1j * 4.0 * x[2]) * (1.0 + 0.5 * n[0]) + x[0] * x[1]

    for kind in (("DP", 0), ("P", 1)):
        ref_space = bempp_cl.api.function_space(ref_grid, *kind)
        ref = bempp_cl.api.GridFunction(ref_space, fun=fun).projections(ref_space)
        got = project_callable_device(_device_fun(), function_space(ours, *kind)).cpu().numpy()
        assert _rel(got, ref) < 1e-12, kind
