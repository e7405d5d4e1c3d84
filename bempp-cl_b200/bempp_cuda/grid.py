"""Triangle surface grids: geometry and element adjacency.

The attribute names and array layouts follow ``bempp_cl.api.grid.grid.Grid``
(bempp_cl/api/grid/grid.py:15-140, :552-590) so that a space or assembler
written against the reference can read either class:

* ``vertices``  float64 (3, nv), ``elements`` uint32 (3, ne)
* ``jacobians`` float64 (ne, 3, 2) with columns v1 - v0 and v2 - v0
* ``normals`` (ne, 3) unit normals, ``integration_elements`` (ne,) = 2 * area
* ``jacobian_inverse_transposed`` (ne, 3, 2) = J (J^T J)^-1
* ``edge_adjacency`` int32 (6, E): e0, e1, then local vertex indices of the
  shared edge in e0 (two values) and in e1 (two values, ascending)
* ``vertex_adjacency`` int32 (4, V): e0, e1, local index of the shared vertex
  in e0 and in e1

Both orderings (e0, e1) and (e1, e0) of an adjacent pair are listed, as in the
reference (grid.py:510-550, :1048-1100).  The local vertex index convention of
the shared edge decides which remapped Sauter-Schwab rule a pair gets, so it
is reproduced exactly: the shared vertices are found by scanning e0's local
vertices in order, then both pairs are swapped if that leaves e1's indices
descending (grid.py:1026-1045).
"""

import numpy as _np

# Local vertex pairs of the three local edges (grid.py:12).
EDGE_LOCAL = _np.array([[0, 1], [2, 0], [1, 2]], dtype=_np.int64)


class Grid(object):
    """A flat-triangle surface grid with precomputed geometry."""

    _next_id = 0

    def __init__(self, vertices, elements, domain_indices=None):
        vertices = _np.asarray(vertices, dtype=_np.float64)
        elements = _np.asarray(elements)
        if vertices.ndim != 2 or vertices.shape[0] != 3:
            raise ValueError("vertices must have shape (3, number_of_vertices)")
        if elements.ndim != 2 or elements.shape[0] != 3:
            raise ValueError("elements must have shape (3, number_of_elements)")
        if elements.size and (elements.min() < 0 or elements.max() >= vertices.shape[1]):
            raise ValueError("element vertex index out of range")
        if not _np.all(_np.isfinite(vertices)):
            raise ValueError("vertices must be finite")
        self._vertices = _np.asfortranarray(vertices)
        self._elements = _np.asfortranarray(elements.astype(_np.uint32))
        ne = self._elements.shape[1]
        if domain_indices is None:
            domain_indices = _np.zeros(ne, dtype=_np.uint32)
        self._domain_indices = _np.asarray(domain_indices, dtype=_np.uint32)
        Grid._next_id += 1
        self._id = "cudagrid_%d" % Grid._next_id

        self._compute_geometry()
        self._enumerate_edges()
        self._compute_adjacency()
        self._vertex_neighbors = None
        self._edge_neighbors = None
        self._device_cache = {}

    # ------------------------------------------------------------------ geometry
    def _compute_geometry(self):
        """Per-element Jacobians, normals and integration elements (grid.py:552-590)."""
        v = self._vertices
        e = self._elements.astype(_np.int64)
        v0 = v[:, e[0]].T
        v1 = v[:, e[1]].T
        v2 = v[:, e[2]].T
        j0 = v1 - v0
        j1 = v2 - v0
        cross = _np.cross(j0, j1)
        norms = _np.linalg.norm(cross, axis=1)
        if _np.any(norms == 0.0):
            bad = int(_np.flatnonzero(norms == 0.0)[0])
            raise ValueError("degenerate element %d (zero area)" % bad)
        self._normals = cross / norms[:, None]
        self._volumes = 0.5 * norms
        self._jacobians = _np.stack([j0, j1], axis=2)  # (ne, 3, 2)
        jtj = _np.einsum("eki,ekj->eij", self._jacobians, self._jacobians)
        det = jtj[:, 0, 0] * jtj[:, 1, 1] - jtj[:, 0, 1] * jtj[:, 1, 0]
        self._integration_elements = _np.sqrt(det)
        inv = _np.empty_like(jtj)
        inv[:, 0, 0] = jtj[:, 1, 1] / det
        inv[:, 1, 1] = jtj[:, 0, 0] / det
        inv[:, 0, 1] = -jtj[:, 0, 1] / det
        inv[:, 1, 0] = -jtj[:, 1, 0] / det
        self._jac_inv_trans = _np.einsum("eki,eij->ekj", self._jacobians, inv)
        self._centroids = (v0 + v1 + v2) / 3.0
        diff = _np.linalg.norm(j0 - j1, axis=1)
        self._diameters = _np.linalg.norm(j0, axis=1) * _np.linalg.norm(j1, axis=1) * diff / norms

    def _enumerate_edges(self):
        """Number edges in order of first appearance (grid.py:1408-1440)."""
        e = self._elements.astype(_np.int64)
        ne = e.shape[1]
        a = e[EDGE_LOCAL[:, 0]]  # (3, ne)
        b = e[EDGE_LOCAL[:, 1]]
        lo = _np.minimum(a, b).T.reshape(-1)  # element-major, local edge minor
        hi = _np.maximum(a, b).T.reshape(-1)
        key = lo * (int(self._vertices.shape[1]) + 1) + hi
        uniq, first, inverse = _np.unique(key, return_index=True, return_inverse=True)
        # renumber unique edges by first appearance
        order = _np.argsort(first, kind="stable")
        rank = _np.empty_like(order)
        rank[order] = _np.arange(len(order))
        edge_index = rank[inverse]
        self._element_edges = _np.asfortranarray(edge_index.reshape(ne, 3).T.astype(_np.uint32))
        edges = _np.empty((2, len(uniq)), dtype=_np.uint32)
        edges[0, edge_index] = lo
        edges[1, edge_index] = hi
        self._edges = edges

    def _compute_adjacency(self):
        """Edge- and vertex-adjacent ordered element pairs with local indices."""
        from scipy.sparse import csr_matrix

        e = self._elements.astype(_np.int64)
        ne = e.shape[1]
        nv = self._vertices.shape[1]
        incidence = csr_matrix(
            (_np.ones(3 * ne, dtype=_np.int32), (e.T.reshape(-1), _np.repeat(_np.arange(ne), 3))),
            shape=(nv, ne),
        )
        shared = (incidence.T @ incidence).tocoo()
        rows = shared.row.astype(_np.int64)
        cols = shared.col.astype(_np.int64)
        count = shared.data
        offdiag = rows != cols
        order = _np.lexsort((cols, rows))
        rows, cols, count, offdiag = rows[order], cols[order], count[order], offdiag[order]

        # eq[k, i, j]: local vertex i of element rows[k] equals local vertex j of cols[k]
        def matches(r, c):
            return e[:, r].T[:, :, None] == e[:, c].T[:, None, :]

        vsel = offdiag & (count == 1)
        r, c = rows[vsel], cols[vsel]
        eq = matches(r, c)
        flat = eq.reshape(len(r), 9).argmax(axis=1)
        self._vertex_adjacency = _np.vstack([r, c, flat // 3, flat % 3]).astype(_np.int32)

        esel = offdiag & (count == 2)
        r, c = rows[esel], cols[esel]
        eq = matches(r, c)
        has = eq.any(axis=2)  # (n, 3): local vertex i of e0 is shared
        jidx = eq.argmax(axis=2)  # matching local index in e1
        # first two shared local indices of e0 in scan order
        i_sorted = _np.argsort(~has, axis=1, kind="stable")[:, :2]
        i0 = i_sorted[:, 0]
        i1 = i_sorted[:, 1]
        n = len(r)
        j0 = jidx[_np.arange(n), i0]
        j1 = jidx[_np.arange(n), i1]
        swap = j1 < j0
        a0 = _np.where(swap, i1, i0)
        a1 = _np.where(swap, i0, i1)
        b0 = _np.where(swap, j1, j0)
        b1 = _np.where(swap, j0, j1)
        self._edge_adjacency = _np.vstack([r, c, a0, a1, b0, b1]).astype(_np.int32)

    # --------------------------------------------------------------- properties
    @property
    def id(self):
        return self._id

    @property
    def vertices(self):
        return self._vertices

    @property
    def elements(self):
        return self._elements

    @property
    def domain_indices(self):
        return self._domain_indices

    @property
    def number_of_vertices(self):
        return self._vertices.shape[1]

    @property
    def number_of_elements(self):
        return self._elements.shape[1]

    @property
    def number_of_edges(self):
        return self._edges.shape[1]

    @property
    def edges(self):
        return self._edges

    @property
    def element_edges(self):
        return self._element_edges

    @property
    def normals(self):
        return self._normals

    @property
    def volumes(self):
        return self._volumes

    @property
    def jacobians(self):
        return self._jacobians

    @property
    def jacobian_inverse_transposed(self):
        return self._jac_inv_trans

    @property
    def integration_elements(self):
        return self._integration_elements

    @property
    def centroids(self):
        return self._centroids

    @property
    def diameters(self):
        return self._diameters

    @property
    def edge_adjacency(self):
        return self._edge_adjacency

    @property
    def vertex_adjacency(self):
        return self._vertex_adjacency

    @property
    def vertex_on_boundary(self):
        """True for vertices on an edge that has only one element."""
        counts = _np.bincount(self._element_edges.ravel(), minlength=self.number_of_edges)
        out = _np.zeros(self.number_of_vertices, dtype=bool)
        out[self._edges[:, counts == 1].ravel()] = True
        return out

    @property
    def edge_neighbors(self):
        """For each edge the tuple of adjacent elements in increasing order."""
        if self._edge_neighbors is None:
            ee = self._element_edges.astype(_np.int64)
            ne = ee.shape[1]
            flat_edges = ee.T.reshape(-1)
            flat_elems = _np.repeat(_np.arange(ne), 3)
            order = _np.lexsort((flat_elems, flat_edges))
            starts = _np.searchsorted(flat_edges[order], _np.arange(self.number_of_edges + 1))
            el = flat_elems[order]
            self._edge_neighbors = [tuple(el[starts[k] : starts[k + 1]]) for k in range(self.number_of_edges)]
        return self._edge_neighbors

    @property
    def vertex_neighbors(self):
        """CSR (indices, indexptr) of the elements around each vertex."""
        if self._vertex_neighbors is None:
            e = self._elements.astype(_np.int64)
            ne = e.shape[1]
            flat_v = e.T.reshape(-1)
            flat_e = _np.repeat(_np.arange(ne), 3)
            order = _np.lexsort((flat_e, flat_v))
            ptr = _np.searchsorted(flat_v[order], _np.arange(self.number_of_vertices + 1))
            self._vertex_neighbors = (flat_e[order].astype(_np.uint32), ptr.astype(_np.uint32))
        return self._vertex_neighbors

    def local2global(self, element, local_points):
        """Map (2, n) reference points of one element to (3, n) global points."""
        return self._vertices[:, self._elements[0, element]][:, None] + self._jacobians[element] @ local_points

    def __eq__(self, other):
        return isinstance(other, Grid) and other.id == self.id

    def __hash__(self):
        return hash(self._id)
