"""Distribution of a dense operator over ranks (one process per GPU).

Symmetric stripes (``stripe_bounds``, ``assemble_stripe``,
``StripeOperator``; the default for one DP0 space on both sides): rank r
sweeps the element pairs (i, j), i <= j, with rows i in its stripe
[lo_r, hi_r), the stripes cut so that every rank has the same number of
pairs.  It keeps A_ij in U_r and the transposed entries A_ji in L_r, both
(hi_r - lo_r) x (n - lo_r): each pair's kernel work is done once for both
entries on any number of ranks, and the ranks together hold n^2 entries.
The singular pairs go to the rank that owns the smaller element.  The
matvec is U_r x[lo:] on the stripe's rows plus L_r^T x[lo:hi] on rows lo..n,
one all-gather of the iterate and one all-reduce of the product.

Row blocks (``row_block``, ``assemble_row_block``, ``RowBlockOperator``):
rank r assembles every entry of a contiguous block of rows (a DP0 dual space
restricted to the block, so the singular pairs it computes are those whose
test element it owns), entry by entry: a pair across two blocks is
evaluated by both ranks; its matvec needs only the all-gather.

Neither assembly communicates.  A distributed solve needs, per GMRES
iteration, the matvec's collectives and one all-reduce per
orthogonalisation step and per norm; the small Hessenberg system is
replicated on every rank.  torch.distributed supplies the collectives: NCCL
between GPUs, gloo on CPU (tests).

The reference solves on one host with scipy (api/linalg/iterative_solvers.py:47-93)
and has no distributed dense path; the partition helpers here also serve the
batched launch, which shards whole problems over ranks by work.
"""

import numpy as _np
import torch as _torch


def row_block(n, world, rank):
    """Rows [lo, hi) of rank ``rank`` when ``n`` rows are split into ``world`` contiguous blocks."""
    return (n * rank) // world, (n * (rank + 1)) // world


def shard_problems(sizes, world, rank):
    """Indices of the problems of this rank: largest first onto the least-loaded rank (load = n^2)."""
    load = [0] * world
    mine = []
    for i in sorted(range(len(sizes)), key=lambda j: (-sizes[j], j)):
        r = min(range(world), key=lambda j: (load[j], j))
        load[r] += sizes[i] ** 2
        if r == rank:
            mine.append(i)
    return sorted(mine)


def allreduce_sum(tensor, group=None):
    """Sum ``tensor`` over the ranks in place and return it (complex tensors as real pairs)."""
    import torch.distributed as dist

    view = _torch.view_as_real(tensor) if tensor.is_complex() else tensor
    dist.all_reduce(view, op=dist.ReduceOp.SUM, group=group)
    return tensor


class RowBlockOperator(object):
    """Rows [lo, hi) of an n x n matrix held by this rank; matvec on row-distributed vectors."""

    def __init__(self, local_rows, n, world, rank, group=None):
        self.local_rows = local_rows
        self.n = int(n)
        self.world = int(world)
        self.rank = int(rank)
        self.group = group
        self.blocks = [row_block(self.n, self.world, r) for r in range(self.world)]
        lo, hi = self.blocks[self.rank]
        if tuple(local_rows.shape) != (hi - lo, self.n):
            raise ValueError("rank %d holds rows [%d, %d) of %d columns; got %s"
                             % (self.rank, lo, hi, self.n, tuple(local_rows.shape)))
        self.width = max(h - l for l, h in self.blocks)

    @property
    def local_range(self):
        return self.blocks[self.rank]

    def gather(self, x_local):
        """The full vector from every rank's block (one all-gather of equal, padded blocks)."""
        import torch.distributed as dist

        pad = _torch.zeros(self.width, dtype=x_local.dtype, device=x_local.device)
        pad[: x_local.shape[0]] = x_local
        parts = [_torch.empty_like(pad) for _ in range(self.world)]
        if pad.is_complex():
            dist.all_gather([_torch.view_as_real(p) for p in parts], _torch.view_as_real(pad), group=self.group)
        else:
            dist.all_gather(parts, pad, group=self.group)
        return _torch.cat([parts[r][: h - l] for r, (l, h) in enumerate(self.blocks)])

    def matvec(self, x_local):
        return _torch.mv(self.local_rows, self.gather(x_local))

    def allreduce(self, tensor):
        return allreduce_sum(tensor, self.group)


def gmres_distributed(op, b_local, tol=1e-8, restart=100, maxiter=None):
    """GMRES on row-distributed vectors; returns (x_local, info, residuals, iterations) on every rank."""
    from .linalg import gmres_tensor

    return gmres_tensor(op.matvec, b_local, tol=tol, restart=restart, maxiter=maxiter, allreduce=op.allreduce,
                        global_size=op.n)


def assemble_row_block(grid, descriptor, world, rank, parameters=None, precision=None, diag_shift=0.0,
                       symmetric=True):
    """The rows of this rank of a DP0 x DP0 operator on ``grid`` as a device tensor (no communication)."""
    from . import _lib
    from .assembly import regular_into, singular_into_dense
    from .operators import Parameters
    from .space import function_space

    parameters = parameters or Parameters()
    domain = function_space(grid, "DP", 0)
    n = grid.number_of_elements
    lo, hi = row_block(n, world, rank)
    dual = domain if (lo, hi) == (0, n) else function_space(grid, "DP", 0, support_elements=_np.arange(lo, hi))
    dtype = _torch.complex128 if descriptor.is_complex else _torch.float64
    out = _torch.empty((hi - lo, n), dtype=dtype, device="cuda")
    regular_into(out, descriptor, domain, dual, parameters, precision=_lib.FP64 if precision is None else precision,
                 overwrite=True, symmetric=symmetric)
    singular_into_dense(out, descriptor, domain, dual, parameters, diag_shift=diag_shift)
    return out


# --------------------------------------------------------------------------------- symmetric stripes
def stripe_bounds(n, world):
    """Row boundaries lo_0 = 0 < lo_1 < ... < lo_world = n of equal upper-triangle work: rows [0, b) hold
    b n - b (b - 1) / 2 pairs (i, j), i <= j."""
    total = n * (n + 1) / 2.0
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        # b n - b (b - 1) / 2 = target  <=>  b^2 - (2 n + 1) b + 2 target = 0 (the smaller root)
        b = ((2 * n + 1) - _np.sqrt((2 * n + 1) ** 2 - 8.0 * target)) / 2.0
        bounds.append(int(min(max(round(b), bounds[-1]), n)))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


class _StripeSingular(object):
    """The singular pairs (t, s) with min(t, s) in [lo, hi) of one DP0 space on the device, with their
    places in the stripe: t <= s at U[t - lo, s - lo], t > s at L[s - lo, t - lo] (the entry A_ts)."""

    def __init__(self, space, order, lo, hi):
        from .device import DeviceSingularRule, singular_rule_arrays

        arrays = singular_rule_arrays(space.grid, order, space.support, space.support)
        te = _np.asarray(arrays[3], dtype=_np.int64)
        se = _np.asarray(arrays[4], dtype=_np.int64)
        low = _np.minimum(te, se)
        sel = _np.flatnonzero((low >= lo) & (low < hi))
        self.count = int(sel.size)
        self.rule = DeviceSingularRule(list(arrays[:3]) + [_np.asarray(a)[sel] for a in arrays[3:]]) \
            if sel.size else None
        t, s_ = te[sel], se[sel]
        upper = t <= s_
        rows = _torch.as_tensor(_np.where(upper, t, s_) - lo, device="cuda")
        cols = _torch.as_tensor(_np.where(upper, s_, t) - lo, device="cuda")
        up = _torch.as_tensor(upper, device="cuda")
        self.upper = (rows[up], cols[up], up)
        self.lower = (rows[~up], cols[~up], ~up)


def _stripe_plan(space, order, lo, hi):
    from .device import _cache

    cache = _cache(space.grid)
    key = ("stripe_singular", _torch.cuda.current_device(), int(order), int(lo), int(hi))
    if key not in cache:
        cache[key] = _StripeSingular(space, order, lo, hi)
    return cache[key]


def stripe_singular_pairs(space, parameters, lo, hi):
    """Number of singular pairs the stripe [lo, hi) of one DP0 space owns."""
    return _stripe_plan(space, parameters.quadrature.singular, lo, hi).count


def singular_into_stripe(U, L, lo, hi, descriptor, space, parameters, diag_shift=0.0):
    """Add the singular (adjacent) pairs (t, s) with min(t, s) in [lo, hi) of one DP0 space: t <= s into
    U[t - lo, s - lo], t > s into L[s - lo, t - lo] (the entry A_ts), and diag_shift * |e| at (e, e).
    The pair values come from the library's singular kernel (one value per pair); the pair list of
    the stripe is built once per grid and stripe."""
    from . import _lib
    from .assembly import _set_params, kernel_ids
    from .device import current_stream, device_grid, device_space, ptr

    grid = space.grid
    plan = _stripe_plan(space, parameters.quadrature.singular, lo, hi)
    if plan.count:
        kernel, assembly = kernel_ids(descriptor)
        values = _torch.zeros(plan.count, dtype=U.dtype, device=U.device)
        args = _lib.SingularArgs()
        args.kernel = kernel
        args.assembly = assembly
        args.is_complex = 1 if values.is_complex() else 0
        _set_params(args, descriptor.options)
        args.grid = device_grid(grid).record()
        args.test = args.trial = device_space(space).record()
        plan.rule.fill(args)
        args.values = ptr(values)
        args.dense = None
        args.ld = 0
        args.diag_shift = 0.0
        _lib.check(_lib.load().bemppcuda_assemble_singular(args, current_stream()))
        rows, cols, up = plan.upper
        U.index_put_((rows, cols), values[up], accumulate=True)
        rows, cols, low = plan.lower
        L.index_put_((rows, cols), values[low], accumulate=True)
    if diag_shift != 0.0:
        idx = _torch.arange(hi - lo, device=U.device)
        areas = _torch.as_tensor(_np.asarray(grid.volumes)[lo:hi], device=U.device, dtype=_torch.float64)
        U[idx, idx] += (diag_shift * areas).to(U.dtype)


def stripe_entries(n, lo, hi):
    """Matrix entries a stripe holds: both entries of every pair (i, j), lo <= i < hi, i < j, and (i, i)."""
    pairs = (hi - lo) * n - (lo + hi - 1) * (hi - lo) // 2
    return 2 * pairs - (hi - lo)


def assemble_stripe(grid, descriptor, world, rank, parameters=None, precision=None, diag_shift=0.0, out=None):
    """(U, L, (lo, hi)) of this rank for a DP0 x DP0 operator on ``grid`` (no communication).

    ``out`` = (U, L) reuses buffers of a previous call (their entries with j < i stay zero)."""
    from . import _lib
    from .assembly import regular_into
    from .operators import Parameters
    from .space import function_space

    parameters = parameters or Parameters()
    space = function_space(grid, "DP", 0)
    n = grid.number_of_elements
    lo, hi = stripe_bounds(n, world)[rank]
    if out is None:
        dtype = _torch.complex128 if descriptor.is_complex else _torch.float64
        U = _torch.zeros((hi - lo, n - lo), dtype=dtype, device="cuda")
        L = _torch.zeros_like(U)
    else:
        U, L = out
    if hi > lo:
        regular_into(U, descriptor, space, space, parameters,
                     precision=_lib.FP64 if precision is None else precision, overwrite=True, rows=(lo, hi),
                     tresult=L, col_begin=lo)
        singular_into_stripe(U, L, lo, hi, descriptor, space, parameters, diag_shift)
    return U, L, (lo, hi)


class StripeOperator(object):
    """This rank's stripe (U, L) of an n x n matrix; matvec on row-distributed vectors (rank r holds
    rows [lo_r, hi_r) of ``stripe_bounds``)."""

    def __init__(self, U, L, n, world, rank, group=None, allreduce=None, allgather=None):
        self.U, self.L = U, L
        self.n, self.world, self.rank = int(n), int(world), int(rank)
        self.group = group
        self.blocks = stripe_bounds(self.n, self.world)
        lo, hi = self.blocks[self.rank]
        if tuple(U.shape) != (hi - lo, self.n - lo) or U.shape != L.shape:
            raise ValueError("rank %d holds stripe [%d, %d) of %d columns; got %s / %s"
                             % (self.rank, lo, hi, self.n, tuple(U.shape), tuple(L.shape)))
        self.width = max(h - l for l, h in self.blocks)
        self._allreduce = allreduce
        self._allgather = allgather

    @property
    def local_range(self):
        return self.blocks[self.rank]

    def gather(self, x_local):
        if self._allgather is not None:
            return self._allgather(x_local)
        return RowBlockOperator.gather(self, x_local)

    def allreduce(self, tensor):
        if self._allreduce is not None:
            return self._allreduce(tensor)
        return allreduce_sum(tensor, self.group)

    def partial_product(self, x):
        """This rank's share of A x for the full vector x (nonzero on rows lo .. n)."""
        from .matmat import matvec_of

        lo, hi = self.local_range
        y = _torch.zeros(self.n, dtype=_torch.promote_types(self.U.dtype, x.dtype), device=x.device)
        if hi > lo:
            xt = x[lo:].to(y.dtype)
            y[lo:hi] += matvec_of(self.U.to(y.dtype) if self.U.dtype != y.dtype else self.U)(xt)
            y[lo:] += _torch.mv(self.L.transpose(0, 1).to(y.dtype), x[lo:hi].to(y.dtype))
        return y

    def matvec(self, x_local):
        lo, hi = self.local_range
        y = self.allreduce(self.partial_product(self.gather(x_local)))
        return y[lo:hi]
