"""Batched DP0 assembly: many grids and wavenumbers in one persistent launch.

``BatchAssembler`` assembles, for a list of grids and wavenumbers, the DP0
Helmholtz single-layer (or the combined field DLP + eta SLP + c I) weak form of
every problem with ONE persistent regular-pair launch over all (problem,
tile) work items and ONE singular launch over the concatenated pair lists
(csrc/batch.cu).  The reference has no batched path: it assembles one
operator per ``weak_form()`` (core/dense_assembler.py:49-98), so a batch of 64
is 64 separate assemblies there.

* ``launch()`` queues device work only (counter reset and two kernels) and can
  be captured in a CUDA graph: ``capture()`` records launch (plus, optionally,
  the multi-right-hand-side products of all problems, one batched launch of
  csrc/matmat.cu) into a ``torch.cuda.CUDAGraph`` and ``replay()`` runs it.
* ``autotune()`` times the launch for candidate tile shapes (test rows per
  work item) and persistent grid sizes (CTAs per SM) and keeps the fastest;
  results are cached per (kernel, precision mix, work-size bucket) in
  memory and, when ``BEMPP_CUDA_TUNE_CACHE`` names a file, on disk.
"""

import ctypes as _ct
import json as _json
import math as _math
import os as _os

import numpy as _np
import torch as _torch

from . import _lib
from .assembly import regular_rule
from .device import current_stream, device_grid, device_space, ptr, require_cuda, singular_rule_arrays
from .matmat import BatchedProduct
from .shapes import ellipsoid
from .space import function_space

_TUNE_MEMO = {}
ROW_CANDIDATES = (8, 16, 32)
BPS_CANDIDATES = (2, 3, 4, 5, 6, 8)


def c4_problems(count=64, seed=0, levels=(3, 4, 5), kmin=1.0, kmax=16.0):
    """Seeded batch of ellipsoids: regular_sphere(L) scaled by semi-axes U[0.5, 1.5], k ~ U[kmin, kmax]."""
    rng = _np.random.default_rng(seed)
    out = []
    for _ in range(count):
        level = int(rng.choice(levels))
        axes = rng.uniform(0.5, 1.5, size=3)
        k = float(rng.uniform(kmin, kmax))
        out.append((ellipsoid(level, *axes), k))
    return out


class BatchAssembler(object):
    """Device matrices of many DP0 Helmholtz problems assembled in one launch."""

    def __init__(self, grids, wavenumbers, precision="fp64", kernel="helmholtz_single_layer", eta=None,
                 identity=0.0, rows_per_item=32, blocks_per_sm=4, parameters=None):
        require_cuda()
        if len(grids) != len(wavenumbers) or not grids:
            raise ValueError("one wavenumber per grid is required")
        if kernel not in ("helmholtz_single_layer", "helmholtz_combined_field"):
            raise ValueError("batched kernels: helmholtz_single_layer, helmholtz_combined_field")
        precisions = [precision] * len(grids) if isinstance(precision, str) else list(precision)
        order_reg = parameters.quadrature.regular if parameters is not None else 4
        order_sing = parameters.quadrature.singular if parameters is not None else 4
        if int(order_reg) != 4:
            raise ValueError("the batched kernel uses the 6-point rule (regular order 4)")
        self.kernel = kernel
        self.grids = list(grids)
        self.wavenumbers = [complex(k) for k in wavenumbers]
        self.precisions = precisions
        self.spaces = [function_space(g, "DP", 0) for g in self.grids]
        self.outputs = [
            _torch.empty((g.number_of_elements, g.number_of_elements), dtype=_torch.complex128, device="cuda")
            for g in self.grids
        ]
        self._problems = (_lib.BatchProblem * len(grids))()
        te, se, toff, soff, woff, npts = [], [], [], [], [], []
        tables = None
        begin = 0
        for i, (g, sp, k, prec, out) in enumerate(zip(self.grids, self.spaces, self.wavenumbers, precisions,
                                                      self.outputs)):
            dg = device_grid(g)
            ds = device_space(sp)
            arrays = singular_rule_arrays(g, order_sing, sp.support, sp.support)
            if tables is None:
                tables = arrays[:3]
            te.append(arrays[3])
            se.append(arrays[4])
            toff.append(arrays[5])
            soff.append(arrays[6])
            woff.append(arrays[7])
            npts.append(arrays[8])
            p = self._problems[i]
            p.grid = dg.record()
            p.support = ptr(ds.support)
            p.result = ptr(out)
            p.ld = out.stride(0)
            e = complex(eta) if eta is not None else -1j * k
            params = [k.real, k.imag, e.real, e.imag] if kernel == "helmholtz_combined_field" else [k.real, k.imag, 0, 0]
            for j in range(4):
                p.params[j] = float(params[j])
            p.phase_radius = 1.0001 * 2.0 * dg.radius
            p.precision = _lib.MIXED if prec == "mixed" else _lib.FP64
            p.pair_begin = begin
            p.pair_count = len(arrays[3])
            begin += len(arrays[3])
        self.npairs = begin
        dev = lambda a, dt: _torch.as_tensor(_np.ascontiguousarray(a)).to(device="cuda", dtype=dt)
        tp = _np.ascontiguousarray(_np.asarray(tables[0], dtype=_np.float64).T)
        sp_ = _np.ascontiguousarray(_np.asarray(tables[1], dtype=_np.float64).T)
        self._keep = [dev(tp, _torch.float64), dev(sp_, _torch.float64), dev(tables[2], _torch.float64)]
        for arr in (te, se, toff, soff, woff, npts):
            self._keep.append(dev(_np.concatenate(arr).astype(_np.int32), _torch.int32))
        self._qp, self._qw = regular_rule(4)
        nbytes = int(_lib.load().bemppcuda_batch_workspace_bytes(len(grids)))
        self._workspace = _torch.empty(nbytes, dtype=_torch.uint8, device="cuda")
        self.args = _lib.BatchArgs()
        a = self.args
        a.kernel = _lib.KERNEL_IDS[kernel]
        a.nproblems = len(grids)
        a.problems = _ct.cast(self._problems, _ct.POINTER(_lib.BatchProblem))
        a.nq = len(self._qw)
        a.blocks_per_sm = int(blocks_per_sm)
        a.quad_points = self._qp.ctypes.data
        a.quad_weights = self._qw.ctypes.data
        a.npairs = self.npairs
        (a.test_points, a.trial_points, a.weights, a.test_elements, a.trial_elements, a.test_offsets,
         a.trial_offsets, a.weights_offsets, a.npoints) = [ptr(t) for t in self._keep]
        a.diag_shift = float(identity)
        a.rows_per_item = int(rows_per_item)
        a.workspace = ptr(self._workspace)
        a.workspace_bytes = nbytes
        self._graph = None
        self._product = None
        self._product_key = None
        self.prepare()

    @property
    def entries(self):
        return sum(g.number_of_elements ** 2 for g in self.grids)

    def prepare(self):
        _lib.check(_lib.load().bemppcuda_batch_prepare(_ct.byref(self.args), current_stream()))

    def launch(self):
        _lib.check(_lib.load().bemppcuda_batch_launch(_ct.byref(self.args), current_stream()))

    def set_shape(self, rows_per_item, blocks_per_sm):
        self.args.rows_per_item = int(rows_per_item)
        self.args.blocks_per_sm = int(blocks_per_sm)
        self.prepare()  # the tile table depends on rows_per_item
        self._graph = None

    def time_launch(self, repeats=3):
        """Mean device time of one launch in ms (CUDA events on the current stream)."""
        self.launch()
        _torch.cuda.synchronize()
        e0 = _torch.cuda.Event(enable_timing=True)
        e1 = _torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(repeats):
            self.launch()
        e1.record()
        _torch.cuda.synchronize()
        return e0.elapsed_time(e1) / repeats

    def tune_key(self):
        mix = "+".join(sorted(set(self.precisions)))
        bucket = int(_math.log2(max(self.entries, 1)))
        return "%s|%s|%d" % (self.kernel, mix, bucket)

    def autotune(self, rows=ROW_CANDIDATES, blocks=BPS_CANDIDATES, repeats=2):
        """Pick the fastest (rows per work item, CTAs per SM); returns (shape, timings)."""
        key = self.tune_key()
        cache_file = _os.environ.get("BEMPP_CUDA_TUNE_CACHE")
        if key not in _TUNE_MEMO and cache_file and _os.path.exists(cache_file):
            try:
                _TUNE_MEMO.update(_json.load(open(cache_file)))
            except (OSError, ValueError):
                pass
        if key in _TUNE_MEMO:
            shape = tuple(_TUNE_MEMO[key])
            self.set_shape(*shape)
            return shape, {}
        timings = {}
        for r in rows:
            for b in blocks:
                self.set_shape(r, b)
                timings[(r, b)] = self.time_launch(repeats)
        shape = min(timings, key=timings.get)
        self.set_shape(*shape)
        _TUNE_MEMO[key] = list(shape)
        if cache_file:
            try:
                _json.dump(_TUNE_MEMO, open(cache_file, "w"))
            except OSError:
                pass
        return shape, timings

    def step(self, rhs=None, products=None):
        """launch(), then products[i] = outputs[i] @ rhs[i]: the work capture() records, issued eagerly.

        The products of all problems are one batched launch (``matmat.BatchedProduct``);
        its problem table is uploaded on the first call with these tensors.
        """
        self.launch()
        if rhs is not None:
            key = tuple(t.data_ptr() for t in rhs) + tuple(t.data_ptr() for t in products)
            if self._product is None or self._product_key != key:
                if _torch.cuda.is_current_stream_capturing():
                    raise RuntimeError("call step(rhs, products) once before capturing it")
                self._product = BatchedProduct(self.outputs, rhs, products)
                self._product_key = key
            self._product.launch()

    def capture(self, rhs=None, products=None):
        """Record step(rhs, products) in a CUDA graph."""
        self.step(rhs, products)  # warm up outside capture
        _torch.cuda.synchronize()
        graph = _torch.cuda.CUDAGraph()
        with _torch.cuda.graph(graph):
            self.step(rhs, products)
        self._graph = graph
        return graph

    def replay(self):
        if self._graph is None:
            raise RuntimeError("capture() first")
        self._graph.replay()
