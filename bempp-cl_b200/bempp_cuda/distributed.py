"""Row-block distribution of a dense operator over ranks (one process per GPU).

Assembly needs no communication: rank r assembles the rows of a contiguous
block of test elements (a DP0 dual space restricted to that block, so the
singular pairs it computes are those whose test element it owns) and keeps
them in its own HBM.  A distributed solve needs, per GMRES iteration, one
all-gather of the iterate (so every rank can apply its rows to the full
vector) and one all-reduce per orthogonalisation step and per norm; the small
Hessenberg system is replicated on every rank.  torch.distributed supplies the
collectives: NCCL between GPUs, gloo on CPU (tests).

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
