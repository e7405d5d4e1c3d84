"""Row-distributed operator and GMRES on 2 gloo ranks (CPU, no GPU).

Each rank holds a contiguous block of rows of a seeded complex matrix and of
the right-hand side; the distributed GMRES (one all-gather of the iterate per
matvec, all-reduced dot products) must reproduce the single-process solve and
take the same number of iterations on every rank.  Also checks the partition
helpers used by the bench (row blocks, problem shards).
"""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _matrix(n, seed=4):
    rng = np.random.default_rng(seed)
    a = np.eye(n) * 3.0 + (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return a, b


def _worker(rank, world, port, n, restart, result_path):
    import datetime
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "bempp-cl_b200"))
    import torch.distributed as dist

    from bempp_cuda.distributed import RowBlockOperator, gmres_distributed, row_block

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, b = _matrix(n)
        lo, hi = row_block(n, world, rank)
        op = RowBlockOperator(torch.as_tensor(a[lo:hi]), n, world, rank)
        x_local, info, residuals, its = gmres_distributed(op, torch.as_tensor(b[lo:hi]), tol=1e-12, restart=restart)
        full = op.gather(x_local)
        np.savez(result_path % rank, x=full.numpy(), info=info, its=its, res=np.asarray(residuals))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n,restart", [(61, 100), (61, 12)])
def test_distributed_gmres_matches_single_process(tmp_path, n, restart):
    import torch.multiprocessing as mp

    from bempp_cuda.linalg import gmres_tensor

    world = 2
    path = str(tmp_path / "rank%d.npz")
    mp.spawn(_worker, args=(world, _free_port(), n, restart, path), nprocs=world, join=True)
    a, b = _matrix(n)
    x_ref = np.linalg.solve(a, b)
    x1, info1, res1, its1 = gmres_tensor(lambda v: torch.mv(torch.as_tensor(a), v), torch.as_tensor(b), tol=1e-12,
                                         restart=restart)
    outs = [np.load(path % r) for r in range(world)]
    for o in outs:
        assert int(o["info"]) == 0
        assert np.linalg.norm(o["x"] - x_ref) <= 1e-10 * np.linalg.norm(x_ref)
        assert int(o["its"]) == its1  # same Krylov steps as the single-process solve
    assert np.array_equal(outs[0]["x"], outs[1]["x"])
    assert np.allclose(outs[0]["res"], np.asarray(res1), rtol=1e-8, atol=1e-15)


def test_row_blocks_and_problem_shards_partition():
    from bempp_cuda.distributed import row_block, shard_problems

    for n in (1, 7, 32768):
        for world in (1, 2, 3, 8):
            rows = []
            for r in range(world):
                lo, hi = row_block(n, world, r)
                rows.extend(range(lo, hi))
            assert rows == list(range(n))
    sizes = [512] * 14 + [2048] * 25 + [8192] * 25
    for world in (1, 2, 4, 8):
        shards = [shard_problems(sizes, world, r) for r in range(world)]
        assert sorted(i for s in shards for i in s) == list(range(len(sizes)))
        loads = [sum(sizes[i] ** 2 for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(sizes) ** 2


def test_row_block_operator_rejects_wrong_block():
    from bempp_cuda.distributed import RowBlockOperator

    with pytest.raises(ValueError):
        RowBlockOperator(torch.zeros((4, 10)), 10, 2, 0)  # rank 0 of 2 owns rows [0, 5)


def _stripes(a, world, rank):
    """The stripe (U, L) of rank ``rank`` cut from a full matrix, as the stripe assembly leaves it."""
    from bempp_cuda.distributed import stripe_bounds

    n = a.shape[0]
    lo, hi = stripe_bounds(n, world)[rank]
    U = np.zeros((hi - lo, n - lo), dtype=a.dtype)
    L = np.zeros_like(U)
    for i in range(lo, hi):
        U[i - lo, i - lo:] = a[i, i:]       # A_ij, j >= i
        L[i - lo, i + 1 - lo:] = a[i + 1:, i]  # A_ji, j > i
    return U, L


def _stripe_worker(rank, world, port, n, restart, result_path):
    import datetime
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "bempp-cl_b200"))
    import torch.distributed as dist

    from bempp_cuda.distributed import StripeOperator, gmres_distributed, stripe_bounds

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, b = _matrix(n)
        U, L = _stripes(a, world, rank)
        op = StripeOperator(torch.as_tensor(U), torch.as_tensor(L), n, world, rank)
        lo, hi = stripe_bounds(n, world)[rank]
        x = np.random.default_rng(3).standard_normal(n) + 0j
        ax = op.matvec(torch.as_tensor(x[lo:hi]))
        x_local, info, residuals, its = gmres_distributed(op, torch.as_tensor(b[lo:hi]), tol=1e-12, restart=restart)
        full = op.gather(x_local)
        np.savez(result_path % rank, x=full.numpy(), info=info, its=its, ax=ax.numpy(), lo=lo, hi=hi)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_stripe_operator_matvec_and_gmres(tmp_path, world):
    """Symmetric stripes on gloo ranks: the stripe matvec (all-gather + all-reduce) equals A x row by row, and
    the distributed GMRES reproduces the single-process solve."""
    import torch.multiprocessing as mp

    n = 61
    path = str(tmp_path / "stripe%d.npz")
    mp.spawn(_stripe_worker, args=(world, _free_port(), n, 30, path), nprocs=world, join=True)
    a, b = _matrix(n)
    x = np.random.default_rng(3).standard_normal(n) + 0j
    x_ref = np.linalg.solve(a, b)
    for r in range(world):
        o = np.load(path % r)
        lo, hi = int(o["lo"]), int(o["hi"])
        np.testing.assert_allclose(o["ax"], (a @ x)[lo:hi], rtol=0, atol=1e-12 * np.abs(a @ x).max())
        assert int(o["info"]) == 0
        assert np.linalg.norm(o["x"] - x_ref) <= 1e-10 * np.linalg.norm(x_ref)


def test_stripe_bounds_balance_the_upper_triangle():
    from bempp_cuda.distributed import stripe_bounds

    for n in (1, 5, 97, 32768):
        for world in (1, 2, 3, 8):
            b = stripe_bounds(n, world)
            assert b[0][0] == 0 and b[-1][1] == n and all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            work = [(h - l) * (n - l) - (h - l) * (h - l - 1) // 2 for l, h in b]
            if n >= 97:
                assert max(work) - min(work) <= n + 1  # within one row of the equal share


def test_stripe_partial_products_sum_to_the_matrix_product():
    """Without collectives: the ranks' partial products of the stripes add up to A x."""
    from bempp_cuda.distributed import StripeOperator

    n = 40
    a, _ = _matrix(n, seed=9)
    x = torch.as_tensor(np.random.default_rng(2).standard_normal(n) + 1j * np.random.default_rng(5).standard_normal(n))
    for world in (1, 2, 4):
        total = torch.zeros(n, dtype=torch.complex128)
        for r in range(world):
            U, L = _stripes(a, world, r)
            total += StripeOperator(torch.as_tensor(U), torch.as_tensor(L), n, world, r).partial_product(x)
        assert np.allclose(total.numpy(), a @ x.numpy(), rtol=0, atol=1e-12)
