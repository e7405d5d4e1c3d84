"""Symmetric stripes of the DP0 sweep (stripe mode of bemppcuda_assemble_regular) on one B200.

The ranks of a multi-GPU run are emulated one after another in one process
(no collectives): their stripes (U, L) must reassemble the matrix of the
ordinary single-GPU assembly (FP64, and mixed precision against mixed), and
the sum of their partial products must equal the full product.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _descriptor(k):
    from bempp_cuda.operators import OperatorDescriptor

    eta = -1j * k
    return OperatorDescriptor("c", [k, 0.0, eta.real, eta.imag], "helmholtz_combined_field", "default_scalar",
                              "double", True, None, 1)


@pytest.mark.parametrize("world", [2, 3, 5])
@pytest.mark.parametrize("mixed", [False, True])
def test_stripes_reassemble_the_matrix(world, mixed):
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.distributed import StripeOperator, assemble_stripe
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import ellipsoid
    from bempp_cuda.space import function_space

    grid = ellipsoid(3, 1.1, 0.9, 0.8)
    n = grid.number_of_elements
    desc = _descriptor(6.0)
    prm = Parameters()
    precision = _lib.MIXED if mixed else _lib.FP64
    sp = function_space(grid, "DP", 0)
    full = torch.empty((n, n), dtype=torch.complex128, device="cuda")
    regular_into(full, desc, sp, sp, prm, precision=precision, overwrite=True)
    singular_into_dense(full, desc, sp, sp, prm, diag_shift=-0.5)
    rebuilt = torch.zeros_like(full)
    x = torch.as_tensor(np.random.default_rng(1).standard_normal(n) + 0j, device="cuda")
    total = torch.zeros(n, dtype=torch.complex128, device="cuda")
    for r in range(world):
        U, L, (lo, hi) = assemble_stripe(grid, desc, world, r, prm, precision=precision, diag_shift=-0.5)
        for i in range(lo, hi):
            rebuilt[i, i:] += U[i - lo, i - lo:]
            rebuilt[i + 1:, i] += L[i - lo, i + 1 - lo:]
        total += StripeOperator(U, L, n, world, r).partial_product(x)
    err = (torch.linalg.norm(rebuilt - full) / torch.linalg.norm(full)).item()
    assert err < 1e-14, err
    ref = torch.mv(full, x)
    assert (torch.linalg.norm(total - ref) / torch.linalg.norm(ref)).item() < 1e-13


def test_stripe_mode_rejects_non_symmetric_sweeps():
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(1)
    sp = function_space(grid, "DP", 0)
    U = torch.zeros((4, 32), dtype=torch.complex128, device="cuda")
    with pytest.raises(_lib.BemppCudaError):  # a stripe needs a row range
        regular_into(U, _descriptor(2.0), sp, sp, Parameters(), overwrite=True, tresult=torch.zeros_like(U))
