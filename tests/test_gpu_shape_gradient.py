"""Adjoint shape gradient of the far-field objective (run on a B200).

* forward pieces (A, b, u, J) against the oracle on the host;
* each of the three contractions of the adjoint kernel against central
  differences of the quantity it differentiates, on every coordinate of a
  small grid;
* the full gradient (vertices and k) against central differences of J with
  h = 1e-6 on 20 seeded coordinates, on the device objective and on the host
  (oracle) objective;
* the torch.autograd.Function wrapper.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

H = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _objective(level, seed=0, k=6.0, ndir=32):
    from bempp_cuda.shape_gradient import FarFieldObjective, fibonacci_directions
    from bempp_cuda.shapes import perturbed_sphere

    grid, _ = perturbed_sphere(level, seed=seed)
    return FarFieldObjective(grid, directions=fibonacci_directions(ndir)), k


def _coords(nv, count, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(nv * 3, size=count, replace=False)
    return [(int(f) // 3, int(f) % 3) for f in flat]


def _fd(fun, x0, v, c, h=H):
    xp = x0.clone()
    xm = x0.clone()
    xp[v, c] += h
    xm[v, c] -= h
    return (fun(xp) - fun(xm)) / (2.0 * h)


def test_forward_matches_oracle():
    from shape_oracle import host_objective

    obj, k = _objective(2)
    verts = obj.vertices
    value, state = obj.evaluate(verts, k, keep=True)
    geo = state.geometry
    a_dev = obj.assemble(geo, k).cpu().numpy()
    b_dev = obj.rhs(geo, k).cpu().numpy()
    j_host, a_host, b_host, u_host = host_objective(verts.cpu().numpy(), obj.base.elements.cpu().numpy(), k,
                                                    obj.directions.cpu().numpy())
    assert np.linalg.norm(a_dev - a_host) <= 1e-12 * np.linalg.norm(a_host)
    assert np.linalg.norm(b_dev - b_host) <= 1e-13 * np.linalg.norm(b_host)
    u_dev = state.u.cpu().numpy()
    assert np.linalg.norm(u_dev - u_host) <= 1e-10 * np.linalg.norm(u_host)
    assert abs(value.item() - j_host) <= 1e-10 * j_host


@pytest.mark.parametrize("term", ["operator", "farfield", "rhs"])
def test_each_contraction_against_central_differences(term):
    """Every coordinate of a level-1 grid: kernel contraction vs FD of the contracted quantity."""
    obj, k = _objective(1, seed=3)
    x0 = obj.vertices.clone()
    value, state = obj.evaluate(x0, k, keep=True)
    rng = np.random.default_rng(5)
    n = obj.base.nelements
    lam = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n), device="cuda")
    scales = {"operator": (1.0, 0.0, 0.0), "farfield": (0.0, 1.0, 0.0), "rhs": (0.0, 0.0, 1.0)}[term]
    vgrad, kgrad = obj.gradient(state, k, lam=lam, scales=scales)
    phi, u = state.phi, state.u

    def contracted(x, kk=k):
        geo = obj.geometry(x)
        if term == "operator":
            return torch.real(torch.vdot(lam, obj.assemble(geo, kk) @ phi)).item()
        if term == "farfield":
            return torch.real(torch.vdot(u, obj.farfield_matrix(geo, kk) @ phi)).item()
        return torch.real(torch.vdot(lam, obj.rhs(geo, kk))).item()

    fd = np.zeros((obj.base.nvertices, 3))
    for v in range(obj.base.nvertices):
        for c in range(3):
            fd[v, c] = _fd(contracted, x0, v, c)
    g = vgrad.cpu().numpy()
    assert np.linalg.norm(g - fd) <= 1e-7 * np.linalg.norm(fd), (np.linalg.norm(g - fd), np.linalg.norm(fd))
    fdk = (contracted(x0, k + H) - contracted(x0, k - H)) / (2 * H)
    assert abs(kgrad.item() - fdk) <= 1e-7 * max(abs(fdk), 1e-3 * np.linalg.norm(fd))


@pytest.mark.parametrize("level", [2, 3])
def test_full_gradient_against_central_differences(level):
    obj, k = _objective(level, seed=1)
    x0 = obj.vertices.clone()
    value, state = obj.evaluate(x0, k, keep=True)
    vgrad, kgrad = obj.gradient(state, k)
    coords = _coords(obj.base.nvertices, 20, seed=7)
    fd = np.array([_fd(lambda x: obj.evaluate(x, k).item(), x0, v, c) for v, c in coords])
    ad = np.array([vgrad[v, c].item() for v, c in coords])
    assert np.linalg.norm(ad - fd) <= 1e-6 * np.linalg.norm(fd), (ad, fd)
    fdk = (obj.evaluate(x0, k + H).item() - obj.evaluate(x0, k - H).item()) / (2 * H)
    assert abs(kgrad.item() - fdk) <= 1e-6 * abs(fdk)


@pytest.mark.parametrize("level,count", [(2, 6), (3, 3)])
def test_gradient_against_host_objective_differences(level, count):
    """Central differences of the oracle's J (host assembly, numpy solve) against the device adjoint."""
    from shape_oracle import host_objective

    obj, k = _objective(level, seed=2)
    x0 = obj.vertices.clone()
    value, state = obj.evaluate(x0, k, keep=True)
    vgrad, kgrad = obj.gradient(state, k)
    el = obj.base.elements.cpu().numpy()
    dirs = obj.directions.cpu().numpy()
    x0h = x0.cpu().numpy()
    coords = _coords(obj.base.nvertices, count, seed=11)
    for v, c in coords:
        xp = x0h.copy()
        xm = x0h.copy()
        xp[v, c] += H
        xm[v, c] -= H
        fd = (host_objective(xp, el, k, dirs)[0] - host_objective(xm, el, k, dirs)[0]) / (2 * H)
        assert abs(vgrad[v, c].item() - fd) <= 1e-6 * np.abs(vgrad.cpu().numpy()).max()


def test_autograd_function():
    from bempp_cuda.shape_gradient import far_field_objective

    obj, k = _objective(2, seed=4)
    x = obj.vertices.clone().requires_grad_(True)
    kt = torch.tensor(k, dtype=torch.float64, requires_grad=True)
    j = far_field_objective(x, kt, obj)
    (3.0 * j).backward()
    value, state = obj.evaluate(obj.vertices, k, keep=True)
    vgrad, kgrad = obj.gradient(state, k)
    assert abs(j.item() - value.item()) <= 1e-14 * value.item()
    # the adjoint adds per-element partial sums with FP64 atomics, so two evaluations agree to
    # rounding in summation order (measured ~1e-14 of the largest entry), not bit for bit
    assert torch.allclose(x.grad, 3.0 * vgrad, rtol=1e-12, atol=1e-12 * vgrad.abs().max().item())
    assert abs(kt.grad.item() - 3.0 * kgrad.item()) <= 1e-12 * abs(kgrad.item())


def test_adjoint_rejects_missing_vectors():
    import ctypes

    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream

    obj, k = _objective(1)
    value, state = obj.evaluate(obj.vertices, k, keep=True)
    a = obj._args(state.geometry, k)
    a.scale_operator = 1.0
    vg = torch.zeros((obj.base.nvertices, 3), dtype=torch.float64, device="cuda")
    kg = torch.zeros(1, dtype=torch.float64, device="cuda")
    a.vertex_grad = vg.data_ptr()
    a.k_grad = kg.data_ptr()
    rc = _lib.load().bemppcuda_shape_adjoint_dp0(ctypes.byref(a), current_stream())
    assert rc == _lib.ERR_INVALID and "missing" in _lib.last_error()
    a.nq = 3
    rc = _lib.load().bemppcuda_shape_adjoint_dp0(ctypes.byref(a), current_stream())
    assert rc == _lib.ERR_INVALID and "6-point" in _lib.last_error()
    torch.cuda.synchronize()
    assert not vg.any()


def test_gmres_solver_gives_the_lu_gradient():
    from bempp_cuda.shape_gradient import FarFieldObjective, fibonacci_directions
    from bempp_cuda.shapes import perturbed_sphere

    grid, _ = perturbed_sphere(3, seed=5)
    lu = FarFieldObjective(grid, directions=fibonacci_directions(32))
    it = FarFieldObjective(grid, directions=fibonacci_directions(32), solver="gmres", tol=1e-13)
    v1, s1 = lu.evaluate(lu.vertices, 6.0, keep=True)
    v2, s2 = it.evaluate(it.vertices, 6.0, keep=True)
    g1, k1 = lu.gradient(s1, 6.0)
    g2, k2 = it.gradient(s2, 6.0)
    assert abs(v1.item() - v2.item()) <= 1e-11 * v1.item()
    assert (torch.linalg.norm(g1 - g2) / torch.linalg.norm(g1)).item() <= 1e-9
    assert abs(k1.item() - k2.item()) <= 1e-9 * abs(k1.item())
    assert s2.iterations is not None and s2.iterations > 0


@pytest.mark.parametrize("solver", ["lu32", "gmres32"])
def test_refined_solvers_give_the_lu_gradient(solver):
    """complex64 LU or complex64 GMRES (adjoint through the transposed view), refined in complex128."""
    from bempp_cuda.shape_gradient import FarFieldObjective, fibonacci_directions
    from bempp_cuda.shapes import perturbed_sphere

    grid, _ = perturbed_sphere(3, seed=6)
    lu = FarFieldObjective(grid, directions=fibonacci_directions(32))
    lo = FarFieldObjective(grid, directions=fibonacci_directions(32), solver=solver, tol=1e-13)
    v1, s1 = lu.evaluate(lu.vertices, 6.0, keep=True)
    v2, s2 = lo.evaluate(lo.vertices, 6.0, keep=True)
    g1, k1 = lu.gradient(s1, 6.0)
    g2, k2 = lo.gradient(s2, 6.0)
    assert abs(v1.item() - v2.item()) <= 1e-11 * v1.item()
    assert (torch.linalg.norm(g1 - g2) / torch.linalg.norm(g1)).item() <= 1e-9
    assert abs(k1.item() - k2.item()) <= 1e-9 * abs(k1.item())


def test_gradient_per_coordinate_fourth_order():
    """Every one of 20 seeded coordinates within 1e-6 relative of a fourth-order central difference
    (H = 1e-4; truncation O(H^4)), L3: the per-coordinate bound, which the h = 1e-6 two-point
    difference cannot test on small components (its roundoff eps |J| / h exceeds 1e-6 of them)."""
    obj, k = _objective(3, seed=1)
    x0 = obj.vertices.clone()
    value, state = obj.evaluate(x0, k, keep=True)
    vgrad, _ = obj.gradient(state, k)
    step = 1e-4
    for v, c in _coords(obj.base.nvertices, 20, seed=7):
        vals = []
        for s in (-2, -1, 1, 2):
            xs = x0.clone()
            xs[v, c] += s * step
            vals.append(obj.evaluate(xs, k).item())
        fd4 = (vals[0] - 8 * vals[1] + 8 * vals[2] - vals[3]) / (12 * step)
        assert abs(vgrad[v, c].item() - fd4) <= 1e-6 * abs(fd4), (v, c, vgrad[v, c].item(), fd4)
