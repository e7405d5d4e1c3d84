"""Batched multi-right-hand-side products of dense device operators.

``BatchedProduct(mats, xs, ys)`` computes ``ys[i] = mats[i] @ xs[i]`` for a
list of complex128 device matrices in one kernel launch per group of up to 8
right-hand-side columns (``bemppcuda_matmat_launch``, csrc/matmat.cu).  It is
the device counterpart of DenseDiscreteBoundaryOperator._matmat
(api/assembly/discrete_boundary_operator.py:192-198), which multiplies one
host matrix at a time; here the operators stay where they were assembled and
a list of them (the batched assembly's outputs, each with its own right-hand
sides) costs one launch instead of one library GEMM per operator.

The problem table is uploaded once by the constructor; ``launch()`` queues
device work only and can be captured in a CUDA graph.  Two to eight
right-hand sides run on the FP64 tensor cores.

``gemv(a, x)`` is the one-right-hand-side product y = A x of the solves
(``bemppcuda_gemv``): complex128 or complex64 row-major matrices, streamed
from HBM by the library's own kernel.
"""

import ctypes as _ct

import torch as _torch

from . import _lib
from .device import current_stream, ptr, require_cuda

MAX_RHS = 8


def _check_operand(t, name, i):
    if not isinstance(t, _torch.Tensor) or t.dim() != 2:
        raise ValueError("%s[%d] must be a 2-D tensor" % (name, i))
    if t.dtype != _torch.complex128:
        raise ValueError("%s[%d] must be complex128 (got %s)" % (name, i, t.dtype))
    if t.stride(1) != 1 or t.stride(0) < t.shape[1]:
        raise ValueError("%s[%d] must have unit column stride (row-major rows)" % (name, i))


def validate(mats, xs, ys):
    """Shapes, dtypes and strides of the operand lists; returns the right-hand-side count."""
    if not (len(mats) == len(xs) == len(ys)) or not mats:
        raise ValueError("mats, xs and ys must be non-empty lists of equal length")
    nrhs = None
    for i, (a, x, y) in enumerate(zip(mats, xs, ys)):
        _check_operand(a, "mats", i)
        _check_operand(x, "xs", i)
        _check_operand(y, "ys", i)
        m, n = a.shape
        if m == 0 or n == 0:
            raise ValueError("mats[%d] is empty" % i)
        if x.shape[0] != n or y.shape[0] != m or x.shape[1] != y.shape[1]:
            raise ValueError("problem %d: shapes %s @ %s -> %s do not match"
                             % (i, tuple(a.shape), tuple(x.shape), tuple(y.shape)))
        if nrhs is None:
            nrhs = x.shape[1]
        elif x.shape[1] != nrhs:
            raise ValueError("every problem needs the same number of right-hand sides")
    if nrhs == 0:
        raise ValueError("no right-hand sides")
    for name, lst in (("mats", mats), ("xs", xs), ("ys", ys)):
        for i, t in enumerate(lst):
            if t.device.type != "cuda":
                raise ValueError("%s[%d] must be a CUDA tensor" % (name, i))
    return nrhs


class BatchedProduct(object):
    """ys[i] = mats[i] @ xs[i] (complex128, device) in one launch per 8 right-hand-side columns."""

    def __init__(self, mats, xs, ys):
        require_cuda()
        nrhs = validate(mats, xs, ys)
        self.mats, self.xs, self.ys = list(mats), list(xs), list(ys)  # keep the storage alive
        self._chunks = []
        lib = _lib.load()
        for c0 in range(0, nrhs, MAX_RHS):
            nr = min(MAX_RHS, nrhs - c0)
            probs = (_lib.MatmatProblem * len(mats))()
            for i, (a, x, y) in enumerate(zip(mats, xs, ys)):
                p = probs[i]
                p.a = a.data_ptr()
                p.x = x.data_ptr() + 16 * c0
                p.y = y.data_ptr() + 16 * c0
                p.rows, p.cols = a.shape
                p.lda, p.ldx, p.ldy = a.stride(0), x.stride(0), y.stride(0)
            nbytes = int(lib.bemppcuda_matmat_workspace_bytes(len(mats)))
            ws = _torch.empty(nbytes, dtype=_torch.uint8, device="cuda")
            args = _lib.MatmatArgs()
            args.nproblems = len(mats)
            args.nrhs = nr
            args.problems = _ct.cast(probs, _ct.POINTER(_lib.MatmatProblem))
            args.workspace = ptr(ws)
            args.workspace_bytes = nbytes
            _lib.check(lib.bemppcuda_matmat_prepare(_ct.byref(args), current_stream()))
            self._chunks.append((args, probs, ws))

    @property
    def entries(self):
        return sum(a.shape[0] * a.shape[1] for a in self.mats)

    def launch(self):
        lib = _lib.load()
        for args, _, _ in self._chunks:
            _lib.check(lib.bemppcuda_matmat_launch(_ct.byref(args), current_stream()))


def matmat(mats, xs, ys=None):
    """ys[i] = mats[i] @ xs[i] for lists of complex128 device tensors; returns ys."""
    if ys is None:
        ys = [_torch.empty((a.shape[0], x.shape[1]), dtype=_torch.complex128, device=a.device)
              for a, x in zip(mats, xs)]
    BatchedProduct(mats, xs, ys).launch()
    return ys


def gemv(a, x, out=None, stream=None):
    """y = a @ x for a complex128 / complex64 device matrix with unit column stride and a vector of
    the same dtype (bemppcuda_gemv); ``out`` (rows,) receives the result when given."""
    require_cuda()
    if a.dim() != 2 or a.dtype not in (_torch.complex128, _torch.complex64):
        raise ValueError("gemv: a must be a 2-D complex128 or complex64 tensor (got %s)" % (a.dtype,))
    if a.stride(1) != 1 or (a.shape[0] > 1 and a.stride(0) < a.shape[1]):
        raise ValueError("gemv: a must have unit column stride (row-major rows)")
    if x.dim() != 1 or x.shape[0] != a.shape[1]:
        raise ValueError("gemv: x must be a vector of length %d" % a.shape[1])
    x = x.to(a.dtype).contiguous()
    if out is None:
        out = _torch.empty(a.shape[0], dtype=a.dtype, device=a.device)
    elif out.dtype != a.dtype or not out.is_contiguous() or out.shape != (a.shape[0],):
        raise ValueError("gemv: out must be a contiguous (rows,) tensor of the matrix dtype")
    lda = a.stride(0) if a.shape[0] > 1 else a.shape[1]
    _lib.check(_lib.load().bemppcuda_gemv(ptr(a), a.shape[0], a.shape[1], lda, ptr(x), ptr(out),
                                          1 if a.dtype == _torch.complex64 else 0, stream or current_stream()))
    return out


def matvec_of(a):
    """v -> a @ v: the library GEMV for complex device matrices; torch.mv for real ones and for host
    tensors (the solvers' host-side tests and tools; the product path's matrices are on the device)."""
    if a.is_cuda and a.is_complex() and a.stride(1) == 1:
        return lambda v: gemv(a, v)
    return lambda v: _torch.mv(a, v)
