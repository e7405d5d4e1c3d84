"""Batched multi-right-hand-side products (csrc/matmat.cu) against torch.matmul (run on a B200).

The kernel sums in FP64 in its own order, so it agrees with the library
product to rounding: relative Frobenius error <= 1e-14 per problem.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _c128(rng, shape):
    return torch.as_tensor(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), device="cuda")


def _rel(a, b):
    return (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()


@pytest.mark.parametrize("nrhs", [1, 2, 3, 4, 5, 6, 7, 8, 11, 14, 16])
def test_ragged_problems_match_matmul(nrhs):
    """Rectangular and ragged sizes (1 row, 1 column, non-multiples of the 16-row / 64-column tiles);
    more than 8 right-hand sides run as several launches over column groups."""
    from bempp_cuda.matmat import matmat

    rng = np.random.default_rng(nrhs)
    shapes = [(1, 1), (17, 5), (130, 64), (64, 130), (1000, 999), (2048, 2048), (3, 4097)]
    mats = [_c128(rng, s) for s in shapes]
    xs = [_c128(rng, (s[1], nrhs)) for s in shapes]
    ys = matmat(mats, xs)
    torch.cuda.synchronize()
    for a, x, y in zip(mats, xs, ys):
        assert _rel(y, a @ x) < 1e-14


def test_strided_views_and_overwrite():
    """Row strides larger than the row (views into wider buffers); ys is overwritten, its padding untouched."""
    from bempp_cuda.matmat import BatchedProduct

    rng = np.random.default_rng(5)
    big_a = _c128(rng, (300, 700))
    big_x = _c128(rng, (700, 12))
    big_y = torch.full((300, 12), 7.0 + 7.0j, dtype=torch.complex128, device="cuda")
    a, x, y = big_a[10:250, 20:620], big_x[20:620, 2:6], big_y[10:250, 3:7]
    bp = BatchedProduct([a], [x], [y])
    for _ in range(2):  # repeated launches give the same result (no accumulation)
        bp.launch()
    torch.cuda.synchronize()
    assert _rel(y, a @ x) < 1e-14
    mask = torch.ones_like(big_y, dtype=torch.bool)
    mask[10:250, 3:7] = False
    assert bool((big_y[mask] == 7.0 + 7.0j).all())


@pytest.mark.parametrize("nrhs", [2, 4, 6, 8])
def test_aligned_and_unaligned_rows(nrhs):
    """The same matrix at a 32-byte aligned address (rows read with 32-byte loads), 16 bytes past it
    and with an odd row stride (16-byte loads): all three agree with the library product, and the
    two 16-byte forms with each other bit for bit."""
    from bempp_cuda.matmat import BatchedProduct

    rng = np.random.default_rng(40 + nrhs)
    rows, cols = 300, 1000
    base = torch.zeros(rows * (cols + 2) + 4, dtype=torch.complex128, device="cuda")
    assert base.data_ptr() % 32 == 0
    src = _c128(rng, (rows, cols))
    views = [
        base[: rows * cols].view(rows, cols),  # aligned, lda even
        base[1 : 1 + rows * (cols + 2)].view(rows, cols + 2)[:, :cols],  # 16 bytes off, lda even
        base[2 : 2 + rows * (cols + 1)].view(rows, cols + 1)[:, :cols],  # aligned, lda odd
    ]
    x = _c128(rng, (cols, nrhs))
    ref = src @ x
    outs = []
    for a in views:
        a.copy_(src)
        y = torch.empty((rows, nrhs), dtype=torch.complex128, device="cuda")
        BatchedProduct([a], [x], [y]).launch()
        torch.cuda.synchronize()
        assert _rel(y, ref) < 1e-14
        outs.append(y)
    assert torch.equal(outs[1], outs[2])


def test_nearly_real_products():
    """Gauss's form (5 to 8 right-hand sides) keeps the normwise bound when the product is almost
    real: the imaginary part's error stays at rounding level relative to |A| |X|."""
    from bempp_cuda.matmat import matmat

    rng = np.random.default_rng(9)
    a = torch.as_tensor(rng.standard_normal((512, 512)) + 1e-9j * rng.standard_normal((512, 512)), device="cuda")
    x = torch.as_tensor(rng.standard_normal((512, 8)) + 1e-9j * rng.standard_normal((512, 8)), device="cuda")
    (y,) = matmat([a], [x])
    torch.cuda.synchronize()
    ref = a @ x
    scale = (a.abs() @ x.abs()).max().item()
    assert (y - ref).abs().max().item() < 1e-13 * scale


def test_graph_capture_of_products():
    from bempp_cuda.matmat import BatchedProduct

    rng = np.random.default_rng(6)
    mats = [_c128(rng, (n, n)) for n in (128, 512, 96)]
    xs = [_c128(rng, (n, 8)) for n in (128, 512, 96)]
    ys = [torch.empty_like(x) for x in xs]
    bp = BatchedProduct(mats, xs, ys)
    bp.launch()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        bp.launch()
    for x in xs:
        x.mul_(2.0)
    g.replay()
    torch.cuda.synchronize()
    for a, x, y in zip(mats, xs, ys):
        assert _rel(y, a @ x) < 1e-14


def test_library_rejects_bad_tables():
    import ctypes

    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream, ptr

    a = torch.zeros((4, 4), dtype=torch.complex128, device="cuda")
    x = torch.zeros((4, 2), dtype=torch.complex128, device="cuda")
    y = torch.zeros((4, 2), dtype=torch.complex128, device="cuda")
    probs = (_lib.MatmatProblem * 1)()
    p = probs[0]
    p.a, p.x, p.y = a.data_ptr(), x.data_ptr(), y.data_ptr()
    p.rows, p.cols, p.lda, p.ldx, p.ldy = 4, 4, 4, 2, 2
    lib = _lib.load()
    ws = torch.empty(int(lib.bemppcuda_matmat_workspace_bytes(1)), dtype=torch.uint8, device="cuda")
    args = _lib.MatmatArgs(nproblems=1, nrhs=9, problems=ctypes.cast(probs, ctypes.POINTER(_lib.MatmatProblem)),
                           workspace=ptr(ws), workspace_bytes=ws.numel())
    assert lib.bemppcuda_matmat_prepare(ctypes.byref(args), current_stream()) == _lib.ERR_INVALID
    args.nrhs = 2
    p.lda = 3  # shorter than a row
    assert lib.bemppcuda_matmat_prepare(ctypes.byref(args), current_stream()) == _lib.ERR_INVALID
    p.lda = 4
    p.x = x.data_ptr() + 8  # not 16-byte aligned
    assert lib.bemppcuda_matmat_prepare(ctypes.byref(args), current_stream()) == _lib.ERR_INVALID
    assert "aligned" in _lib.last_error()
    p.x = x.data_ptr()
    args.workspace_bytes = 0
    assert lib.bemppcuda_matmat_prepare(ctypes.byref(args), current_stream()) == _lib.ERR_WORKSPACE
    args.workspace_bytes = ws.numel()
    assert lib.bemppcuda_matmat_prepare(ctypes.byref(args), current_stream()) == _lib.OK
    assert args.blocks == 1


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(1, 1), (3, 200), (257, 129), (1000, 4097), (4096, 4096)])
def test_gemv_matches_mv(dtype, shape):
    """The solves' one-right-hand-side product (bemppcuda_gemv) = torch.mv to rounding: 1e-14 relative
    (complex128) / 1e-6 (complex64), ragged sizes around the 4-row / 128-column steps."""
    from bempp_cuda.matmat import gemv

    rng = np.random.default_rng(shape[0] + shape[1])
    a = _c128(rng, shape).to(dtype)
    x = _c128(rng, (shape[1],)).to(dtype)
    y = gemv(a, x)
    ref = torch.mv(a.to(torch.complex128), x.to(torch.complex128))
    assert y.dtype == dtype
    assert _rel(y.to(torch.complex128), ref) < (1e-14 if dtype == torch.complex128 else 1e-6)


def test_gemv_strided_rows_and_operator_dot():
    """Row stride wider than the row (a view), and DenseDeviceOperator @ vector taking this path."""
    from bempp_cuda.matmat import gemv
    from bempp_cuda.operators import DenseDeviceOperator

    rng = np.random.default_rng(9)
    big = _c128(rng, (400, 900))
    a = big[7:307, 11:611]
    x = _c128(rng, (600,))
    out = torch.empty(300, dtype=torch.complex128, device="cuda")
    gemv(a, x, out=out)
    assert _rel(out, a @ x) < 1e-14
    op = DenseDeviceOperator(big.contiguous())
    v = _c128(rng, (900,))
    assert _rel(op @ v, big @ v) < 1e-14
    with pytest.raises(ValueError):
        gemv(big.transpose(0, 1), v)
