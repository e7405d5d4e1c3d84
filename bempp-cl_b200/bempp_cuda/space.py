"""Function spaces on a ``Grid``: DP0, DP1, P1, RWG and SNC.

Each space exposes the attributes that the dense assembly path reads from
``bempp_cl.api.space.space.FunctionSpace`` (bempp_cl/api/space/space.py:283-460):
``local2global`` uint32 (ne, nshape), ``local_multipliers`` float64
(ne, nshape), ``normal_multipliers`` int32 (ne,), ``support`` bool (ne,),
``support_elements``, ``number_of_shape_functions``, ``shapeset.identifier``,
``global_dof_count``, ``localised_space`` and ``get_elements_by_color``.

Dof numbering follows the reference so that matrices agree entry by entry:

* DP0 / DP1: support elements in increasing order, nshape dofs each
  (scalar_spaces.py:11-60, :122-166).
* P1: one dof per vertex that touches the support, numbered by vertex index
  (scalar_spaces.py:339-430).
* RWG / SNC: one dof per interior edge, numbered in order of first visit over
  support elements and local edges; the multiplier is +1 on the lower-index
  element of the edge and -1 on the other (maxwell_spaces.py:545-620).  SNC
  shares the RWG dof map and reference shape functions (shapesets.py:151-157).
"""

import numpy as _np


class Shapeset(object):
    """Reference shape functions: identifier and count (shapesets.py:46-158)."""

    _COUNT = {"p0_discontinuous": 1, "p1_discontinuous": 3, "rwg0": 3, "snc0": 3}

    def __init__(self, identifier):
        if identifier not in self._COUNT:
            raise ValueError("unknown shapeset %r" % identifier)
        self.identifier = identifier
        self.number_of_shape_functions = self._COUNT[identifier]

    def evaluate(self, local_coordinates):
        """Values (codomain, nshape, npoints) of the reference functions."""
        x = _np.asarray(local_coordinates, dtype=_np.float64)
        n = x.shape[1]
        if self.identifier == "p0_discontinuous":
            return _np.ones((1, 1, n))
        if self.identifier == "p1_discontinuous":
            return _np.stack([1.0 - x[0] - x[1], x[0], x[1]])[None]
        vals = _np.empty((2, 3, n))
        vals[0] = _np.vstack([x[0], x[0] - 1.0, x[0]])
        vals[1] = _np.vstack([x[1] - 1.0, x[1], x[1]])
        return vals


class FunctionSpace(object):
    """A discrete function space over a grid (no dof transformation)."""

    def __init__(
        self,
        grid,
        identifier,
        shapeset,
        codomain_dimension,
        local2global,
        local_multipliers,
        support,
        normal_multipliers,
        is_localised,
    ):
        self.grid = grid
        self.identifier = identifier
        self.shapeset = Shapeset(shapeset)
        self.codomain_dimension = codomain_dimension
        self.local2global = _np.ascontiguousarray(local2global, dtype=_np.uint32)
        self.local_multipliers = _np.ascontiguousarray(local_multipliers, dtype=_np.float64)
        self.support = _np.asarray(support, dtype=bool)
        self.normal_multipliers = _np.asarray(normal_multipliers, dtype=_np.int32)
        self.support_elements = _np.flatnonzero(self.support).astype(_np.uint32)
        self.number_of_support_elements = len(self.support_elements)
        self.grid_dof_count = int(self.local2global[self.support].max()) + 1 if self.number_of_support_elements else 0
        self.global_dof_count = self.grid_dof_count
        self.requires_dof_transformation = False
        self.is_barycentric = False
        self._is_localised = is_localised
        self._localised = None
        self._colors = None

    @property
    def number_of_shape_functions(self):
        return self.shapeset.number_of_shape_functions

    @property
    def is_localised(self):
        return self._is_localised

    @property
    def localised_space(self):
        """Space with one dof per (support element, local function), multipliers 1."""
        if self._is_localised:
            return self
        if self._localised is None:
            nshape = self.number_of_shape_functions
            ne = self.grid.number_of_elements
            l2g = _np.zeros((ne, nshape), dtype=_np.uint32)
            l2g[self.support] = _np.arange(nshape * self.number_of_support_elements).reshape(-1, nshape)
            mult = _np.zeros((ne, nshape))
            mult[self.support] = 1.0
            self._localised = FunctionSpace(
                self.grid,
                self.identifier + "_localised",
                self.shapeset.identifier,
                self.codomain_dimension,
                l2g,
                mult,
                self.support,
                self.normal_multipliers,
                True,
            )
        return self._localised

    @property
    def map_to_full_grid(self):
        """Sparse (nshape * ne, grid_dof_count) map from dofs to element-local values."""
        from scipy.sparse import coo_matrix

        nshape = self.number_of_shape_functions
        sup = self.support_elements.astype(_np.int64)
        rows = nshape * _np.repeat(sup, nshape) + _np.tile(_np.arange(nshape), len(sup))
        cols = self.local2global[sup].ravel()
        vals = self.local_multipliers[sup].ravel()
        return coo_matrix(
            (vals, (rows, cols)), shape=(nshape * self.grid.number_of_elements, self.grid_dof_count)
        ).tocsr()

    @property
    def dof_transformation(self):
        from scipy.sparse import identity

        return identity(self.global_dof_count, dtype=_np.float64, format="csr")

    def get_elements_by_color(self):
        """Support elements sorted by a colouring in which no two elements of a
        colour share a dof (space.py:612-733).  Returns (indices, indexptr)."""
        if self._colors is None:
            nshape = self.number_of_shape_functions
            sup = self.support_elements.astype(_np.int64)
            dof_elems = {}
            for e in sup:
                for k in range(nshape):
                    if self.local_multipliers[e, k] != 0:
                        dof_elems.setdefault(int(self.local2global[e, k]), []).append(int(e))
            color = -_np.ones(self.grid.number_of_elements, dtype=_np.int64)
            for e in sup:
                taken = set()
                for k in range(nshape):
                    if self.local_multipliers[e, k] != 0:
                        for other in dof_elems[int(self.local2global[e, k])]:
                            if other != e and color[other] >= 0:
                                taken.add(int(color[other]))
                c = 0
                while c in taken:
                    c += 1
                color[e] = c
            ncolors = int(color.max()) + 1 if len(sup) else 0
            indices = _np.concatenate([_np.flatnonzero(color == c) for c in range(ncolors)]).astype(_np.uint32)
            indexptr = _np.zeros(ncolors + 1, dtype=_np.uint32)
            indexptr[1:] = _np.cumsum([_np.count_nonzero(color == c) for c in range(ncolors)])
            self._colors = (indices, indexptr)
        return self._colors

    def __eq__(self, other):
        return (
            isinstance(other, FunctionSpace)
            and other.grid == self.grid
            and other.shapeset.identifier == self.shapeset.identifier
            and _np.array_equal(other.local2global, self.local2global)
            and _np.array_equal(other.local_multipliers, self.local_multipliers)
            and _np.array_equal(other.normal_multipliers, self.normal_multipliers)
        )

    def __hash__(self):
        return id(self)


def _normal_multipliers(grid, swapped_normals):
    nm = _np.ones(grid.number_of_elements, dtype=_np.int32)
    if swapped_normals:
        for k, d in enumerate(grid.domain_indices):
            if d in swapped_normals:
                nm[k] = -1
    return nm


def _support(grid, support_elements, segments):
    if support_elements is not None and segments is not None:
        raise ValueError("Only one of 'support_elements' and 'segments' must be nonzero.")
    ne = grid.number_of_elements
    if support_elements is not None:
        s = _np.zeros(ne, dtype=bool)
        s[_np.asarray(support_elements, dtype=_np.int64)] = True
        return s
    if segments is not None:
        return _np.isin(grid.domain_indices, list(segments))
    return _np.ones(ne, dtype=bool)


def _dp_space(grid, nshape, shapeset, ident, support, nm):
    sup = _np.flatnonzero(support)
    l2g = _np.zeros((grid.number_of_elements, nshape), dtype=_np.uint32)
    l2g[sup] = _np.arange(nshape * len(sup)).reshape(-1, nshape)
    mult = _np.zeros((grid.number_of_elements, nshape))
    mult[sup] = 1.0
    return FunctionSpace(grid, ident, shapeset, 1, l2g, mult, support, nm, True)


def _p1_space(grid, support, nm):
    """P1 dofs on vertices of the support that are interior to it."""
    e = grid.elements.astype(_np.int64)
    ne = grid.number_of_elements
    nv = grid.number_of_vertices
    # a vertex is a dof when every element around it is in the support and it
    # is not on the grid boundary (include_boundary_dofs=False default)
    unsupported_vertex = _np.zeros(nv, dtype=bool)
    unsupported_vertex[e[:, ~support].ravel()] = True
    is_dof = _np.zeros(nv, dtype=bool)
    is_dof[e[:, support].ravel()] = True
    is_dof &= ~unsupported_vertex & ~grid.vertex_on_boundary
    dof_of_vertex = -_np.ones(nv, dtype=_np.int64)
    dof_of_vertex[is_dof] = _np.arange(_np.count_nonzero(is_dof))
    l2g = _np.zeros((ne, 3), dtype=_np.uint32)
    mult = _np.zeros((ne, 3))
    final_support = _np.zeros(ne, dtype=bool)
    for k in _np.flatnonzero(support):
        d = dof_of_vertex[e[:, k]]
        used = d >= 0
        if not used.any():
            continue
        final_support[k] = True
        mult[k, used] = 1.0
        l2g[k, used] = d[used]
        l2g[k, ~used] = d[used].max()
    return FunctionSpace(grid, "p1_continuous", "p1_discontinuous", 1, l2g, mult, final_support, nm, False)


def _rwg_space(grid, support, nm, shapeset, ident):
    """One dof per edge with two supported neighbours (maxwell_spaces.py:545-620)."""
    ee = grid.element_edges.astype(_np.int64)
    ne = grid.number_of_elements
    neighbors = grid.edge_neighbors
    edge_dof = -_np.ones(grid.number_of_edges, dtype=_np.int64)
    support = support.copy()
    count = 0
    for k in _np.flatnonzero(support):
        has = False
        for loc in range(3):
            edge = ee[loc, k]
            if edge_dof[edge] != -1:
                has = True
                continue
            sup_nb = [n for n in neighbors[edge] if support[n]]
            if len(sup_nb) == 2:
                edge_dof[edge] = count
                count += 1
                has = True
        if not has:
            support[k] = False
    l2g = _np.zeros((ne, 3), dtype=_np.uint32)
    mult = _np.zeros((ne, 3))
    for k in _np.flatnonzero(support):
        dofmap = -_np.ones(3, dtype=_np.int64)
        for loc in range(3):
            edge = ee[loc, k]
            if edge_dof[edge] != -1:
                dofmap[loc] = edge_dof[edge]
                sup_nb = [n for n in neighbors[edge] if support[n]]
                if len(sup_nb) == 1:
                    mult[k, loc] = 1.0
                else:
                    mult[k, loc] = 1.0 if k == min(sup_nb) else -1.0
        first = 0
        for loc in range(3):
            if mult[k, loc] != 0:
                first = loc
                break
        for loc in range(3):
            if mult[k, loc] == 0:
                dofmap[loc] = dofmap[first]
        l2g[k] = dofmap
    return FunctionSpace(grid, ident, shapeset, 3, l2g, mult, support, nm, False)


def function_space(grid, kind, degree, support_elements=None, segments=None, swapped_normals=None):
    """Create a space: ("DP", 0), ("DP", 1), ("P", 1), ("RWG", 0), ("SNC", 0)."""
    support = _support(grid, support_elements, segments)
    nm = _normal_multipliers(grid, swapped_normals)
    key = (kind, degree)
    if key == ("DP", 0):
        return _dp_space(grid, 1, "p0_discontinuous", "p0_discontinuous", support, nm)
    if key == ("DP", 1):
        return _dp_space(grid, 3, "p1_discontinuous", "p1_discontinuous", support, nm)
    if key == ("P", 1):
        return _p1_space(grid, support, nm)
    if key == ("RWG", 0):
        return _rwg_space(grid, support, nm, "rwg0", "rwg0")
    if key == ("SNC", 0):
        return _rwg_space(grid, support, nm, "snc0", "snc0")
    raise ValueError("unsupported space %r" % (key,))
