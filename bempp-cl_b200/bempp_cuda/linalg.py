"""Dense solves on the device: GMRES, multi-right-hand-side GMRES and FP64 refinement.

``gmres`` mirrors ``bempp_cl.api.linalg.gmres`` (api/linalg/iterative_solvers.py:47-93):
it takes a boundary operator and a grid function, solves the weak form
against the projections onto the dual space and returns a grid function in
the domain (plus the info code, and optionally residuals / iteration count).
The reference hands the weak form to scipy's GMRES with ``ndarray.dot``
matvecs on the host; here the matrix stays in HBM and every matvec is a
device GEMV (the library's own kernel, bemppcuda_gemv; the batched product for
several right-hand sides); the small orthogonalisation products against the
Krylov basis go through torch (cuBLAS).

``gmres_tensor`` is restarted GMRES on torch tensors: Arnoldi with classical
Gram-Schmidt and one re-orthogonalisation (two GEMVs against the basis per
step instead of j dot products), Givens rotations on the small Hessenberg
system on the host.  Convergence test: ||b - A x|| <= tol ||b|| (the
relative-residual test of scipy's gmres).

``solve_refined`` is mixed-precision iterative refinement: an inner GMRES on
a complex64 copy of the matrix, corrections accumulated in complex128, and
the residual b - A x recomputed in complex128 after every inner solve, until
||b - A x|| <= tol ||b||: with the complex128 matrix, or with the FP64
operator evaluated matrix-free (``operators.fp64_matvec``) when the matrix is
a mixed-precision weak form, so that the iterate converges to the FP64
operator's solution.
"""

import time as _time

import numpy as _np
import torch as _torch


def _norm_t(v, allreduce=None):
    """||v|| as a device scalar (float64), summed over the ranks with ``allreduce``."""
    if allreduce is None:
        return _torch.linalg.vector_norm(v).to(_torch.float64)
    sq = (v.real.square().sum() + v.imag.square().sum()) if v.is_complex() else v.square().sum()
    return _torch.sqrt(allreduce(sq.reshape(1).to(_torch.float64)))[0]


def _norm(v, allreduce=None):
    return float(_norm_t(v, allreduce).item())


class _ArnoldiGraph(object):
    """One Arnoldi step (classical Gram-Schmidt, one re-orthogonalisation) captured in a CUDA graph.

    Shapes are fixed: the step orthogonalises against all restart + 1 rows of
    the basis V, whose rows beyond the current step are zero, so the same
    graph serves every step; the step index lives on the device.  A replay
    reads V[j], writes V[j + 1] and column j of the Hessenberg matrix H and
    advances j.  One launch per step instead of about twenty.
    """

    def __init__(self, matvec, n, restart, dtype, device):
        self.V = _torch.zeros((restart + 1, n), dtype=dtype, device=device)
        self.H = _torch.zeros((restart + 1, restart), dtype=_torch.complex128, device=device)
        self.j = _torch.zeros(1, dtype=_torch.int64, device=device)
        self._rows = _torch.arange(restart + 1, device=device)
        self._matvec = matvec
        side = _torch.cuda.Stream()
        side.wait_stream(_torch.cuda.current_stream())
        with _torch.cuda.stream(side):  # warm-up outside capture (library handles, workspaces)
            self._step()
        _torch.cuda.current_stream().wait_stream(side)
        self.graph = _torch.cuda.CUDAGraph()
        with _torch.cuda.graph(self.graph):
            self._step()

    def _dots(self, w):
        return _torch.mv(self.V.conj(), w)  # V^H w (the conjugate view goes to the GEMV as a flag)

    def _step(self):
        V = self.V
        w = self._matvec(V.index_select(0, self.j).squeeze(0))
        h = self._dots(w)
        w = w - _torch.mv(V.transpose(0, 1), h)
        h2 = self._dots(w)
        w = w - _torch.mv(V.transpose(0, 1), h2)
        hn = _torch.linalg.vector_norm(w).to(_torch.float64)
        V.index_copy_(0, self.j + 1, (w / hn.to(w.dtype)).unsqueeze(0))
        col = (h + h2).to(_torch.complex128) + (self._rows == self.j + 1).to(_torch.complex128) * hn
        self.H.index_copy_(1, self.j, col.unsqueeze(1))
        self.j.add_(1)

    def start(self, v0):
        self.V.zero_()
        self.V[0] = v0
        self.H.zero_()
        self.j.zero_()

    def steps(self, count):
        for _ in range(count):
            self.graph.replay()


def gmres_tensor(matvec, b, x0=None, tol=1e-5, restart=None, maxiter=None, callback=None, allreduce=None,
                 global_size=None, check_every=1, graph=False):
    """Solve A x = b for one right-hand side; return (x, info, residuals, iterations).

    ``matvec(v)`` returns A v for a device vector of b's dtype.  ``info`` is 0
    on convergence, else the number of iterations done (scipy convention).

    ``check_every``: Arnoldi steps run on the device without waiting for the
    host (the Hessenberg columns stay in device memory); every
    ``check_every`` steps the new columns come to the host in one transfer,
    where the Givens rotations give the residual of each step.  The iterate
    and the reported iteration count are those of the first step that meets
    the tolerance; up to ``check_every - 1`` further steps may have been
    computed and are discarded.  1 (default) checks after every step.

    ``graph`` (CUDA tensors, one process): the Arnoldi step is captured once
    in a CUDA graph (``_ArnoldiGraph``; ``matvec`` must be capturable, e.g.
    a GEMV with a fixed matrix) and replayed ``check_every`` times between
    host checks, so the step costs one launch.

    Distributed vectors: when every rank holds a block of rows of b and of the
    iterate, ``allreduce(t)`` must return the sum of ``t`` over the ranks (one
    all-reduce per orthogonalisation step and per norm) and ``matvec`` maps
    the local block of v to the local block of A v (gathering what it needs);
    ``global_size`` caps the restart length.  The small Hessenberg system is
    replicated, so every rank takes the same steps.
    """
    n = b.shape[0] if global_size is None else int(global_size)
    restart = min(restart or 100, n)
    maxiter = maxiter or 10 * n
    check_every = max(1, int(check_every))
    dtype = b.dtype
    red = allreduce if allreduce is not None else (lambda t: t)
    x = _torch.zeros_like(b) if x0 is None else x0.clone()
    bnorm = _norm(b, allreduce)
    residuals = []
    if bnorm == 0.0:
        return x, 0, [0.0], 0
    r = b - matvec(x) if x0 is not None else b.clone()
    beta = _norm(r, allreduce)
    residuals.append(beta / bnorm)
    iterations = 0
    use_graph = bool(graph) and b.is_cuda and allreduce is None
    arnoldi = _ArnoldiGraph(matvec, b.shape[0], restart, dtype, b.device) if use_graph else None
    while True:
        if beta <= tol * bnorm:
            return x, 0, residuals, iterations
        if use_graph:
            arnoldi.start(r / beta)
            V, Hd = arnoldi.V, arnoldi.H
        else:
            V = _torch.empty((restart + 1, b.shape[0]), dtype=dtype, device=b.device)
            V[0] = r / beta
            Hd = _torch.zeros((restart + 1, restart), dtype=_torch.complex128, device=b.device)  # Arnoldi columns
        H = _np.zeros((restart + 1, restart), dtype=_np.complex128)  # rotated (upper triangular)
        cs = _np.zeros(restart, dtype=_np.complex128)
        sn = _np.zeros(restart, dtype=_np.complex128)
        g = _np.zeros(restart + 1, dtype=_np.complex128)
        g[0] = beta
        j_done = 0
        converged = False
        stop = False
        j0 = 0
        while j0 < restart and not stop:
            j1 = min(j0 + check_every, restart, j0 + (maxiter - iterations))
            if use_graph:
                arnoldi.steps(j1 - j0)
            for j in range(j0, j1) if not use_graph else ():
                w = matvec(V[j])
                basis = V[: j + 1]
                h = red(_torch.mv(basis.conj(), w))
                w = w - _torch.mv(basis.transpose(0, 1), h)
                h2 = red(_torch.mv(basis.conj(), w))
                w = w - _torch.mv(basis.transpose(0, 1), h2)
                hn_t = _norm_t(w, allreduce)
                V[j + 1] = w / hn_t.to(w.dtype)  # unused after a breakdown (hn == 0)
                Hd[: j + 1, j] = (h + h2).to(_torch.complex128)
                Hd[j + 1, j] = hn_t.to(_torch.complex128)
            # the new columns reach the host in one transfer
            cols = Hd[: j1 + 1, j0:j1].cpu().numpy()
            for j in range(j0, j1):
                col = _np.zeros(restart + 1, dtype=_np.complex128)
                col[: j + 2] = cols[: j + 2, j - j0]
                hn = float(col[j + 1].real)
                for i in range(j):
                    t = cs[i] * col[i] + sn[i] * col[i + 1]
                    col[i + 1] = -_np.conj(sn[i]) * col[i] + _np.conj(cs[i]) * col[i + 1]
                    col[i] = t
                # rotation G = [[c, s], [-conj(s), conj(c)]] with G (a, b)^T = (rho, 0)^T
                a, bb = col[j], col[j + 1]
                denom = _np.sqrt(abs(a) ** 2 + abs(bb) ** 2)
                if denom == 0.0:
                    cs[j], sn[j] = 1.0, 0.0
                else:
                    cs[j] = _np.conj(a) / denom
                    sn[j] = _np.conj(bb) / denom
                col[j] = denom
                col[j + 1] = 0.0
                H[:, j] = col
                g[j + 1] = -_np.conj(sn[j]) * g[j]
                g[j] = cs[j] * g[j]
                iterations += 1
                j_done = j + 1
                res = abs(g[j + 1])
                residuals.append(res / bnorm)
                if callback is not None:
                    callback(res / bnorm)
                if res <= tol * bnorm or hn == 0.0 or iterations >= maxiter:
                    converged = res <= tol * bnorm or hn == 0.0
                    stop = True
                    break
            j0 = j1
        # solve the triangular system and update x
        y = _np.zeros(j_done, dtype=_np.complex128)
        for i in range(j_done - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1 : j_done] @ y[i + 1 :]) / H[i, i]
        yt = _torch.as_tensor(y, device=b.device).to(dtype if dtype.is_complex else _torch.complex128)
        if not dtype.is_complex:
            yt = yt.real.to(dtype)
        x = x + _torch.mv(V[:j_done].transpose(0, 1), yt)
        if converged:
            return x, 0, residuals, iterations
        if iterations >= maxiter:
            return x, iterations, residuals, iterations
        r = b - matvec(x)
        beta = _norm(r, allreduce)


def gmres_block(matmat, B, tol=1e-5, restart=None, maxiter=None):
    """Several right-hand sides with shared matmats: columns of B (n, m).

    One GMRES per column, but every Arnoldi step multiplies the matrix with
    the basis vectors of all unconverged columns at once (one pass over the
    matrix for m vectors: a GEMM instead of m GEMVs).  Givens rotations per
    column on the host.  Returns (X, infos, iterations per column).
    """
    n, m = B.shape
    restart = min(restart or 100, n)
    maxiter = maxiter or 10 * n
    X = _torch.zeros_like(B)
    bnorms = _torch.linalg.vector_norm(B, dim=0).cpu().numpy()
    iters = _np.zeros(m, dtype=int)
    R = B.clone()
    while True:
        rn = _torch.linalg.vector_norm(R, dim=0).cpu().numpy()
        active = [c for c in range(m) if rn[c] > tol * bnorms[c] and iters[c] < maxiter]
        if not active:
            break
        na = len(active)
        idx = _torch.tensor(active, device=B.device)
        beta = rn[active]
        V = _torch.empty((restart + 1, n, na), dtype=B.dtype, device=B.device)
        V[0] = R[:, idx] / _torch.as_tensor(beta, device=B.device).to(B.dtype)
        H = _np.zeros((na, restart + 1, restart), dtype=_np.complex128)
        cs = _np.zeros((na, restart), dtype=_np.complex128)
        sn = _np.zeros((na, restart), dtype=_np.complex128)
        g = _np.zeros((na, restart + 1), dtype=_np.complex128)
        g[:, 0] = beta
        steps = 0
        for j in range(restart):
            W = matmat(V[j])
            basis = V[: j + 1]
            h = _torch.einsum("kna,na->ka", basis.conj(), W)
            W = W - _torch.einsum("kna,ka->na", basis, h)
            h2 = _torch.einsum("kna,na->ka", basis.conj(), W)
            W = W - _torch.einsum("kna,ka->na", basis, h2)
            hn = _torch.linalg.vector_norm(W, dim=0)
            V[j + 1] = W / _torch.where(hn > 0, hn, _torch.ones_like(hn)).to(B.dtype)
            hcol = (h + h2).to(_torch.complex128).cpu().numpy()  # (j+1, na)
            hnn = hn.to(_torch.float64).cpu().numpy()
            steps = j + 1
            for a in range(na):
                col = _np.zeros(restart + 1, dtype=_np.complex128)
                col[: j + 1] = hcol[:, a]
                col[j + 1] = hnn[a]
                for i in range(j):
                    t = cs[a, i] * col[i] + sn[a, i] * col[i + 1]
                    col[i + 1] = -_np.conj(sn[a, i]) * col[i] + _np.conj(cs[a, i]) * col[i + 1]
                    col[i] = t
                x0, x1 = col[j], col[j + 1]
                den = _np.sqrt(abs(x0) ** 2 + abs(x1) ** 2)
                cs[a, j], sn[a, j] = (1.0, 0.0) if den == 0.0 else (_np.conj(x0) / den, _np.conj(x1) / den)
                col[j], col[j + 1] = den, 0.0
                H[a, :, j] = col
                g[a, j + 1] = -_np.conj(sn[a, j]) * g[a, j]
                g[a, j] = cs[a, j] * g[a, j]
            if all(abs(g[a, j + 1]) <= tol * bnorms[c] for a, c in enumerate(active)) or bool((hnn == 0).all()):
                break
        Y = _np.zeros((steps, na), dtype=_np.complex128)
        for a in range(na):
            for i in range(steps - 1, -1, -1):
                Y[i, a] = (g[a, i] - H[a, i, i + 1 : steps] @ Y[i + 1 :, a]) / H[a, i, i]
        Yt = _torch.as_tensor(Y, device=B.device).to(B.dtype)
        X[:, idx] += _torch.einsum("kna,ka->na", V[:steps], Yt)
        iters[active] += steps
        R = B - matmat(X)
    rn = _torch.linalg.vector_norm(R, dim=0).cpu().numpy()
    infos = [0 if rn[c] <= tol * bnorms[c] else int(iters[c]) for c in range(m)]
    return X, infos, [int(v) for v in iters]


def refine_gmres(matvec, matvec_low, b, tol=1e-8, inner_tol=1e-4, restart=100, maxiter=2000, max_refinements=20,
                 inner_dtype=_torch.complex64, check_every=1):
    """Iterative refinement: inner GMRES with ``matvec_low`` (vectors in ``inner_dtype``), corrections
    and residuals b - A x with ``matvec`` in b's precision; returns (x, info dict)."""
    t0 = _time.perf_counter()
    bnorm = _norm(b)
    x = _torch.zeros_like(b)
    r = b.clone()
    history = []
    inner_iterations = []
    for _ in range(max_refinements):
        res = _norm(r) / bnorm if bnorm > 0.0 else 0.0
        history.append(res)
        if res <= tol:
            break
        d, info, _, its = gmres_tensor(matvec_low, r.to(inner_dtype), tol=inner_tol, restart=restart,
                                       maxiter=maxiter, check_every=check_every)
        inner_iterations.append(its)
        x = x + d.to(b.dtype)
        r = b - matvec(x)
    _torch.cuda.synchronize() if b.is_cuda else None
    info = {
        "refinements": len(inner_iterations),
        "inner_iterations": inner_iterations,
        "relative_residuals": history,
        "converged": history[-1] <= tol,
        "seconds": _time.perf_counter() - t0,
    }
    return x, info


def adjoint_matvec(matrix):
    """v -> A^H v through the transposed view (a GEMV with the transpose flag on the row-major matrix;
    the conjugations touch vectors only, not the matrix)."""
    at = matrix.transpose(0, 1)
    return lambda v: _torch.mv(at, v.conj_physical()).conj_physical()


def solve_refined(matrix, b, tol=1e-8, inner_tol=1e-4, restart=100, maxiter=2000, max_refinements=20,
                  inner_dtype=_torch.complex64, adjoint=False, check_every=1, residual=None):
    """Mixed-precision iterative refinement of A x = b (or A^H x = b); returns (x, info dict).

    ``matrix`` is the (complex128) device matrix; the inner solves use a
    copy in ``inner_dtype``; residuals are formed in complex128, with
    ``residual`` (v -> A v, e.g. operators.fp64_matvec: the FP64 operator
    evaluated matrix-free) when given, else with ``matrix``.  With a mixed
    precision ``matrix`` and the FP64 ``residual`` the iterate converges to
    the FP64 operator's solution; the mixed matrix only preconditions.
    """
    low = matrix.to(inner_dtype)
    b = b.to(matrix.dtype)
    if adjoint:
        if residual is not None:
            raise ValueError("a residual operator is supported for A x = b only")
        hi, lo = adjoint_matvec(matrix), adjoint_matvec(low)
    else:
        from .matmat import matvec_of

        hi = residual if residual is not None else matvec_of(matrix)
        lo = matvec_of(low)
    x, info = refine_gmres(hi, lo, b, tol=tol, inner_tol=inner_tol, restart=restart, maxiter=maxiter,
                           max_refinements=max_refinements, inner_dtype=inner_dtype, check_every=check_every)
    del low
    return x, info


def gmres(A, b, tol=1e-5, restart=None, maxiter=None, use_strong_form=False, return_residuals=False,
          return_iteration_count=False):
    """GMRES on the device for a bempp_cuda boundary operator and grid function."""
    from .grid_function import GridFunction

    if use_strong_form:
        raise ValueError("the strong form is not implemented for the cuda interface")
    mat = A.weak_form()
    rhs = b.projections(A.dual_to_range)
    dtype = mat.tensor.dtype if mat.tensor.is_complex() or not _np.iscomplexobj(rhs) else _torch.complex128
    M = mat.tensor.to(dtype)
    bt = _torch.as_tensor(_np.asarray(rhs)).to(device=M.device, dtype=dtype)
    from .matmat import matvec_of

    x, info, residuals, its = gmres_tensor(matvec_of(M), bt, tol=tol, restart=restart,
                                           maxiter=maxiter)
    sol = GridFunction(A.domain, coefficients=x.cpu().numpy())
    out = [sol, info]
    if return_residuals:
        out.append(residuals)
    if return_iteration_count:
        out.append(its)
    return tuple(out)
