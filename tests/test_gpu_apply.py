"""The matrix-free FP64 operator apply (csrc/apply.cu) against the assembled FP64 weak form (run on a B200).

``operators.fp64_matvec(op, matrix)`` takes the adjacent (singular + identity)
entries from an assembled matrix and evaluates the regular part on the fly;
with the FP64 weak form as ``matrix`` it must reproduce ``A @ x`` to
rounding (1e-13 relative), for every kernel the apply serves, real and
complex wavenumbers (all phase classes), a sphere and an ellipsoid.  With the
mixed-precision matrix it must still give the FP64 product.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _grid(name):
    from bempp_cuda import shapes

    if name == "sphere3":
        return shapes.regular_sphere(3)
    return shapes.ellipsoid(3, 1.3, 0.8, 0.6)


def _ops(sp, k):
    from bempp_cuda import operators

    H, L = operators.boundary.helmholtz, operators.boundary.laplace
    out = {
        "laplace_slp": L.single_layer(sp, sp, sp),
        "laplace_dlp": L.double_layer(sp, sp, sp),
        "laplace_adlp": L.adjoint_double_layer(sp, sp, sp),
        "helmholtz_slp": H.single_layer(sp, sp, sp, k),
        "helmholtz_dlp": H.double_layer(sp, sp, sp, k),
        "helmholtz_adlp": H.adjoint_double_layer(sp, sp, sp, k),
    }
    slp = H.single_layer(sp, sp, sp, k)
    dlp = H.double_layer(sp, sp, sp, k)
    ident = operators.boundary.sparse.identity(sp, sp, sp)
    out["combined"] = dlp - 0.5 * ident - 1j * np.real(k) * slp
    out["combined_scaled"] = 2.0 * dlp + 3.0 * slp
    return out


@pytest.mark.parametrize("grid_name", ["sphere3", "ellipsoid3"])
@pytest.mark.parametrize("k", [2.0, 5.0, 14.0, 4.0 + 1.5j])
def test_apply_equals_assembled_product(grid_name, k):
    from bempp_cuda.operators import fp64_matvec
    from bempp_cuda.space import function_space

    sp = function_space(_grid(grid_name), "DP", 0)
    rng = np.random.default_rng(11)
    n = sp.global_dof_count
    x = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device="cuda")
    for name, op in _ops(sp, k).items():
        if name.startswith("laplace") and k != 2.0:
            continue
        a = op.weak_form().tensor.to(torch.complex128)
        ref = torch.mv(a, x)
        got = fp64_matvec(op, a)(x)
        err = (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item()
        assert err < 1e-13, (name, k, err)


def test_apply_with_mixed_matrix_gives_fp64_product():
    from bempp_cuda import operators
    from bempp_cuda.operators import fp64_matvec
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    k = 10.0
    sp = function_space(regular_sphere(4), "DP", 0)
    H = operators.boundary.helmholtz

    def lhs(interface):
        return (H.double_layer(sp, sp, sp, k, device_interface=interface)
                - 0.5 * operators.boundary.sparse.identity(sp, sp, sp)
                - 1j * k * H.single_layer(sp, sp, sp, k, device_interface=interface))

    a64 = lhs("cuda").weak_form().tensor
    opmx = lhs("cuda_mixed")
    amx = opmx.weak_form().tensor
    x = torch.as_tensor(np.random.default_rng(3).standard_normal(sp.global_dof_count), device="cuda")
    x = x.to(torch.complex128)
    ref = torch.mv(a64, x)
    got = fp64_matvec(opmx, amx)(x)
    assert (torch.linalg.norm(got - ref) / torch.linalg.norm(ref)).item() < 1e-13
    mixed = torch.mv(amx, x)
    assert (torch.linalg.norm(mixed - ref) / torch.linalg.norm(ref)).item() > 1e-12


def test_apply_rejects_unsupported_operators():
    from bempp_cuda import _lib, operators
    from bempp_cuda.operators import fp64_matvec
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    g = regular_sphere(2)
    p1 = function_space(g, "P", 1)
    op = operators.boundary.helmholtz.single_layer(p1, p1, p1, 2.0)
    with pytest.raises((ValueError, _lib.BemppCudaError)):
        fp64_matvec(op, op.weak_form().tensor)(torch.ones(p1.global_dof_count, dtype=torch.complex128,
                                                             device="cuda"))
