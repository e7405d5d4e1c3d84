"""Device-resident copies of grids, spaces and singular rules.

Host objects (``bempp_cuda`` or ``bempp_cl`` grids and spaces, duck-typed)
are uploaded once per CUDA device and cached on the object itself, so a
second assembly on the same grid moves no geometry.  torch is used only for
the allocation and host-to-device copies; every kernel is in libbemppcuda.so.

HBM layout:
* grid: vertices (nv, 3) f64, elements (ne, 3) i32, geometry record
  (25, ne) f64 written by ``bemppcuda_grid_geometry``
* space: support (nsupport,) i32, local2global (ne, nshape) i32, local
  multipliers (ne, nshape) f64, normal multipliers (ne,) i32
* singular rule: point tables (P, 2) f64, weights (W,) f64, six (npairs,)
  i32 pair arrays (test / trial element, three offsets, point count)
"""

import ctypes as _ct

import numpy as _np
import torch as _torch

from . import _lib
from .quadrature import SingularPairs

_CACHE_ATTR = "_bempp_cuda_device_cache"


def require_cuda():
    if not _torch.cuda.is_available():
        raise RuntimeError("bempp_cuda needs a CUDA device (B200, sm_100a); none is visible")
    _lib.load()


def current_stream():
    return _ct.c_void_p(_torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return _ct.c_void_p(t.data_ptr()) if t is not None else None


def _cache(obj):
    cache = getattr(obj, "_bempp_cuda_device_cache_dict", None)
    if cache is None:
        cache = {}
        try:
            setattr(obj, "_bempp_cuda_device_cache_dict", cache)
        except AttributeError:
            pass
    return cache


def to_device(array, dtype):
    return _torch.as_tensor(_np.ascontiguousarray(array)).to(device="cuda", dtype=dtype, non_blocking=False)


def host_grid_arrays(grid):
    """(vertices (nv, 3) f64, elements (ne, 3) i32) in the device layout, from a ``bempp_cuda`` or
    ``bempp_cl`` grid (both store (3, nv) vertices and (3, ne) elements, grid.py:24-60)."""
    vertices = _np.ascontiguousarray(_np.asarray(grid.vertices, dtype=_np.float64).T)
    elements = _np.ascontiguousarray(_np.asarray(grid.elements).T.astype(_np.int32))
    return vertices, elements


def host_space_arrays(space):
    """The host arrays a space uploads, from a ``bempp_cuda`` or ``bempp_cl`` function space
    (space.py:444-459 of the reference): shapeset id, shape count, support (i32), local2global
    (ne, nshape) i32, local multipliers (ne, nshape) f64, normal multipliers (ne,) i32, dof count,
    and whether DP0 dof i is support element i with multiplier 1."""
    nshape = int(space.number_of_shape_functions)
    support = _np.asarray(space.support_elements, dtype=_np.int64)
    l2g = _np.asarray(space.local2global).reshape(-1, nshape)
    mult = _np.asarray(space.local_multipliers, dtype=_np.float64).reshape(-1, nshape)
    ndofs = int(space.global_dof_count)
    pos = (
        nshape == 1
        and len(support) == ndofs
        and _np.array_equal(l2g[support, 0], _np.arange(len(support)))
        and _np.all(mult[support, 0] == 1.0)
    )
    return {
        "shapeset": _lib.SHAPESET_IDS[space.shapeset.identifier],
        "nshape": nshape,
        "support": _np.ascontiguousarray(support.astype(_np.int32)),
        "l2g": _np.ascontiguousarray(l2g.astype(_np.int32)),
        "mult": _np.ascontiguousarray(mult),
        "normal_mult": _np.ascontiguousarray(_np.asarray(space.normal_multipliers, dtype=_np.int32)),
        "ndofs": ndofs,
        "dof_is_position": 1 if pos else 0,
    }


class DeviceGrid(object):
    """Vertices, elements and the per-element geometry record on the device."""

    def __init__(self, grid):
        vertices, elements = host_grid_arrays(grid)
        self.nvertices = vertices.shape[0]
        self.nelements = elements.shape[0]
        self.vertices = to_device(vertices, _torch.float64)
        self.elements = to_device(elements, _torch.int32)
        self.geom = _torch.empty((_lib.GEOM_FIELDS, max(self.nelements, 1)), dtype=_torch.float64, device="cuda")
        _lib.check(
            _lib.load().bemppcuda_grid_geometry(
                ptr(self.vertices),
                self.nvertices,
                ptr(self.elements),
                self.nelements,
                ptr(self.geom),
                current_stream(),
            )
        )
        self.h2d_bytes = vertices.nbytes + elements.nbytes
        # largest centroid-to-vertex distance: bounds every quadrature point's offset from its centroid
        corners = vertices[elements]  # (ne, 3, 3)
        centroids = corners.mean(axis=1, keepdims=True)
        self.radius = float(_np.sqrt(((corners - centroids) ** 2).sum(axis=2)).max()) if self.nelements else 0.0

    def record(self):
        return _lib.GridRec(self.nvertices, self.nelements, ptr(self.geom), ptr(self.elements))


def _shared_on_grid(grid, name, array, dtype):
    """One device copy per distinct content on a grid: spaces with equal maps
    (RWG and SNC on the same grid) get the same device buffers, which is what
    the symmetric sweeps test for."""
    cache = _cache(grid)
    host = _np.ascontiguousarray(array)
    key = ("space_array", _torch.cuda.current_device(), name, str(host.dtype), host.shape, host.tobytes())
    if key not in cache:
        cache[key] = to_device(host, dtype)
    return cache[key]


class DeviceSpace(object):
    """Support list and dof maps of one space on the device."""

    def __init__(self, space):
        h = host_space_arrays(space)
        self.nshape = h["nshape"]
        self.shapeset = h["shapeset"]
        self.nsupport = len(h["support"])
        self.ndofs = h["ndofs"]
        self.dof_is_position = h["dof_is_position"]
        grid = space.grid
        self.support = _shared_on_grid(grid, "support", h["support"], _torch.int32)
        self.l2g = _shared_on_grid(grid, "l2g", h["l2g"], _torch.int32)
        self.mult = _shared_on_grid(grid, "mult", h["mult"], _torch.float64)
        self.normal_mult = _shared_on_grid(grid, "normal_mult", h["normal_mult"], _torch.int32)
        self.h2d_bytes = sum(h[name].nbytes for name in ("support", "l2g", "mult", "normal_mult"))

    def record(self):
        return _lib.Space(
            self.shapeset,
            self.nshape,
            self.nsupport,
            ptr(self.support),
            ptr(self.l2g),
            ptr(self.mult),
            ptr(self.normal_mult),
            self.ndofs,
            self.dof_is_position,
            0,
        )


class DeviceSingularRule(object):
    """Flattened Sauter-Schwab pair list and point tables on the device."""

    def __init__(self, arrays):
        tp, sp, w, te, se, toff, soff, woff, npts = arrays
        tp = _np.ascontiguousarray(_np.asarray(tp, dtype=_np.float64).T)  # (P, 2)
        sp = _np.ascontiguousarray(_np.asarray(sp, dtype=_np.float64).T)
        self.npoints_table = tp.shape[0]
        self.nweights = len(w)
        self.npairs = len(te)
        self.test_points = to_device(tp, _torch.float64)
        self.trial_points = to_device(sp, _torch.float64)
        self.weights = to_device(_np.asarray(w, dtype=_np.float64), _torch.float64)
        ints = [_np.asarray(a).astype(_np.int32) for a in (te, se, toff, soff, woff, npts)]
        (self.test_elements, self.trial_elements, self.test_offsets, self.trial_offsets, self.weights_offsets,
         self.npoints) = [to_device(a, _torch.int32) for a in ints]
        self.h2d_bytes = tp.nbytes + sp.nbytes + 8 * len(w) + sum(a.nbytes for a in ints)
        self._host_ints = ints
        self._by_test = None

    def by_test(self):
        """The pair arrays in test-element order (stable) on the device, and the sorted test elements (host)."""
        if self._by_test is None:
            order = _np.argsort(self._host_ints[0], kind="stable")
            arrays = [to_device(a[order], _torch.int32) for a in self._host_ints]
            self._by_test = (arrays, self._host_ints[0][order])
        return self._by_test

    def pair_range(self, first_element, last_element):
        """[begin, end) of the pairs whose test element lies in [first_element, last_element] (test order)."""
        te_sorted = self.by_test()[1]
        return (int(_np.searchsorted(te_sorted, first_element, "left")),
                int(_np.searchsorted(te_sorted, last_element, "right")))

    def fill(self, args, pairs=None):
        """Point the singular arguments at all pairs, or at pairs [begin, end) of the test-element order."""
        args.npoints_table = self.npoints_table
        args.test_points = ptr(self.test_points)
        args.trial_points = ptr(self.trial_points)
        args.weights = ptr(self.weights)
        args.nweights = self.nweights
        if pairs is None:
            args.npairs = self.npairs
            arrays = (self.test_elements, self.trial_elements, self.test_offsets, self.trial_offsets,
                      self.weights_offsets, self.npoints)
            begin = 0
        else:
            begin, end = pairs
            args.npairs = max(0, end - begin)
            arrays = self.by_test()[0]
        (args.test_elements, args.trial_elements, args.test_offsets, args.trial_offsets, args.weights_offsets,
         args.npoints) = [_ct.c_void_p(a.data_ptr() + 4 * begin) for a in arrays]


def device_grid(grid):
    dev = _torch.cuda.current_device()
    cache = _cache(grid)
    key = ("grid", dev)
    if key not in cache:
        cache[key] = DeviceGrid(grid)
    return cache[key]


def device_space(space):
    dev = _torch.cuda.current_device()
    cache = _cache(space)
    key = ("space", dev)
    if key not in cache:
        cache[key] = DeviceSpace(space)
    return cache[key]


def singular_rule_arrays(grid, order, test_support, trial_support):
    """Host pair arrays of ``grid`` at ``order`` (cached on the grid, like its adjacency)."""
    cache = _cache(grid)
    key = ("singular_host", int(order), _np.asarray(test_support).tobytes(), _np.asarray(trial_support).tobytes())
    if key not in cache:
        cache[key] = SingularPairs(grid, order, test_support, trial_support).arrays()
    return cache[key]


def device_singular_rule(grid, order, test_support, trial_support):
    """Singular pairs of ``grid`` at ``order`` for the given supports, on the device."""
    dev = _torch.cuda.current_device()
    cache = _cache(grid)
    key = ("singular", dev, int(order), _np.asarray(test_support).tobytes(), _np.asarray(trial_support).tobytes())
    if key not in cache:
        cache[key] = DeviceSingularRule(singular_rule_arrays(grid, order, test_support, trial_support))
    return cache[key]


def clear_cache(obj, device_only=False):
    """Drop the device copies (and with ``device_only=False`` the host tables) held for a grid or space."""
    cache = getattr(obj, "_bempp_cuda_device_cache_dict", None)
    if not cache:
        return
    if not device_only:
        cache.clear()
        return
    for key in [k for k in cache if k[0] != "singular_host"]:
        del cache[key]
