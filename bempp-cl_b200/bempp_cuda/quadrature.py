"""Quadrature rules: symmetric triangle rules, Gauss-Legendre and Sauter-Schwab.

* ``triangle_rule(order)`` returns the symmetric triangle rule with the same
  point count per order as ``bempp_cl.api.integration.triangle_gauss.rule``
  (triangle_gauss.py:2928-2940): points (2, n) on the reference triangle
  (0,0), (1,0), (0,1) and weights summing to 1/2.  The rules are the
  published symmetric rules (Strang-Fix / Dunavant); their nodes and weights
  are recomputed here to full double precision by Newton's method on the
  moment equations, seeded with the published 12-15 digit values.
* ``gauss_rule(order)`` is Gauss-Legendre on [0, 1] (gauss.py:1042-1055).
* ``duffy_rule(order, adjacency)`` restates the Sauter-Schwab regularising
  transformations for coincident, edge-adjacent and vertex-adjacent triangle
  pairs (duffy_galerkin.py:25-226; S. Sauter, C. Schwab, "Boundary Element
  Methods", Springer 2011, section 5.2).  The point sets match the reference
  rule point for point; only the order of the points may differ.
* ``SingularPairs`` builds the flattened singular pair list with per-pair
  offsets into one concatenated table of remapped rules, with the layout of
  ``_SingularQuadratureRuleInterfaceGalerkin.get_arrays``
  (core/singular_assembler.py:148-448).
"""

import numpy as _np

# ---------------------------------------------------------------- triangle rules
# Orbit seeds: ("s3", w) | ("s21", a, w) | ("s111", a, b, w); weights relative
# to unit area, barycentric coordinates.
_TRIANGLE_SEEDS = {
    1: [("s3", 1.0)],
    2: [("s21", 1.0 / 6.0, 1.0 / 3.0)],
    3: [("s3", -27.0 / 48.0), ("s21", 0.2, 25.0 / 48.0)],
    4: [("s21", 0.445948490915965, 0.223381589678011), ("s21", 0.091576213509771, 0.109951743655322)],
    5: [
        ("s3", 0.225),
        ("s21", 0.470142064105115, 0.132394152788506),
        ("s21", 0.101286507323456, 0.125939180544827),
    ],
    6: [
        ("s21", 0.249286745170910, 0.116786275726379),
        ("s21", 0.063089014491502, 0.050844906370207),
        ("s111", 0.053145049844817, 0.310352451033784, 0.082851075618374),
    ],
}

_TRIANGLE_DEGREE = {1: 1, 2: 2, 3: 3, 4: 4, 5: 5, 6: 6}


def _orbit_params(seeds):
    params = []
    for orbit in seeds:
        params.extend(orbit[1:])
    return _np.array(params, dtype=_np.float64)


def _expand(seeds, params):
    """Expand orbit parameters into barycentric points (n, 3) and weights."""
    pts, wts = [], []
    k = 0
    for orbit in seeds:
        kind = orbit[0]
        if kind == "s3":
            w = params[k]
            k += 1
            third = (1.0 + 0.0 * w) / 3.0
            pts.append([third, third, third])
            wts.append(w)
        elif kind == "s21":
            a, w = params[k], params[k + 1]
            k += 2
            b = 1.0 - 2.0 * a
            for p in ([a, a, b], [a, b, a], [b, a, a]):
                pts.append(p)
                wts.append(w)
        else:
            a, b, w = params[k], params[k + 1], params[k + 2]
            k += 3
            c = 1.0 - a - b
            for p in ([a, b, c], [a, c, b], [b, a, c], [b, c, a], [c, a, b], [c, b, a]):
                pts.append(p)
                wts.append(w)
    return pts, wts


def _moment_residual(seeds, params, degree):
    pts, wts = _expand(seeds, params)
    res = []
    from math import factorial

    for i in range(degree + 1):
        for j in range(degree + 1 - i):
            exact = factorial(i) * factorial(j) / factorial(i + j + 2) * 2.0  # unit-area normalisation
            s = 0.0
            for p, w in zip(pts, wts):
                s = s + w * p[1] ** i * p[2] ** j
            res.append(s - exact)
    return _np.array(res)


def _solve_rule(order):
    seeds = _TRIANGLE_SEEDS[order]
    degree = _TRIANGLE_DEGREE[order]
    params = _orbit_params(seeds)
    h = 1e-30
    for _ in range(50):
        r = _moment_residual(seeds, params, degree)
        jac = _np.empty((len(r), len(params)))
        for k in range(len(params)):
            step = params.astype(complex)
            step[k] += 1j * h
            jac[:, k] = _moment_residual(seeds, step, degree).imag / h
        delta = _np.linalg.lstsq(jac, -r.real, rcond=None)[0]
        params = params + delta
        if _np.max(_np.abs(delta)) < 1e-17:
            break
    pts, wts = _expand(seeds, params)
    pts = _np.array(pts, dtype=_np.float64)
    points = _np.asfortranarray(_np.vstack([pts[:, 1], pts[:, 2]]))
    return points, 0.5 * _np.array(wts, dtype=_np.float64)


_TRIANGLE_CACHE = {}


def triangle_rule(order):
    """Symmetric triangle quadrature of the given polynomial order."""
    if order not in _TRIANGLE_SEEDS:
        raise ValueError(
            "Symmetric triangle quadrature is available for orders %s; got %r" % (sorted(_TRIANGLE_SEEDS), order)
        )
    if order not in _TRIANGLE_CACHE:
        _TRIANGLE_CACHE[order] = _solve_rule(order)
    p, w = _TRIANGLE_CACHE[order]
    return p.copy(), w.copy()


# ------------------------------------------------------------- Gauss-Legendre
def gauss_rule(order):
    """Gauss-Legendre rule with ``order`` points on [0, 1]."""
    if order < 1 or order > 30:
        raise ValueError("Gauss quadrature order must be between 1 and 30. Provided: %r" % order)
    x, w = _np.polynomial.legendre.leggauss(order)
    # descending nodes, the order of the reference table (gauss.py:1042-1055)
    return 0.5 * (1.0 + x[::-1]), 0.5 * w[::-1]


# ------------------------------------------------------------- Sauter-Schwab
def number_of_duffy_points(order, adjacency):
    """Points per pair: 6 q^4 (coincident), 5 q^4 (edge), 2 q^4 (vertex)."""
    factor = {"coincident": 6, "edge_adjacent": 5, "vertex_adjacent": 2}
    if adjacency not in factor:
        raise ValueError("adjacency must be one of 'coincident', 'edge_adjacent', 'vertex_adjacent'")
    return factor[adjacency] * order**4


def duffy_rule(order, adjacency):
    """Return (test_points (2, n), trial_points (2, n), weights (n,)).

    The four-dimensional cube [0,1]^4 carries a tensor Gauss rule in
    (xi, eta1, eta2, eta3); each region maps the cube onto a piece of the
    product of two triangles and scales the weight by the region's Jacobian.
    The maps are written for the triangle (0,0), (1,0), (1,1) and shifted to
    the reference triangle (0,0), (1,0), (0,1) at the end via x <- x - y.
    """
    x1, w1 = gauss_rule(order)
    n1 = len(x1)
    # tensor order: first coordinate fastest (duffy_galerkin.py:42-50)
    t0 = _np.tile(x1, n1)
    t1 = _np.repeat(x1, n1)
    tw = _np.repeat(w1, n1) * _np.tile(w1, n1)
    nreg = n1 * n1
    # outer loop over the "test" tensor point, inner over the "trial" one
    xi = _np.repeat(t0, nreg)
    e1 = _np.repeat(t1, nreg)
    e2 = _np.tile(t0, nreg)
    e3 = _np.tile(t1, nreg)
    w = _np.repeat(tw, nreg) * _np.tile(tw, nreg)
    e12 = e1 * e2
    e123 = e12 * e3
    one = _np.ones_like(xi)

    if adjacency == "coincident":
        base = w * xi**3 * e1**2 * e2
        regions = [
            ((xi, xi * (1 - e1 + e12)), (xi * (1 - e123), xi * (1 - e1)), base),
            ((xi * (1 - e123), xi * (1 - e1)), (xi, xi * (1 - e1 + e12)), base),
            ((xi, xi * (e1 - e12 + e123)), (xi * (1 - e12), xi * (e1 - e12)), base),
            ((xi * (1 - e12), xi * (e1 - e12)), (xi, xi * (e1 - e12 + e123)), base),
            ((xi * (1 - e123), xi * (e1 - e123)), (xi, xi * (e1 - e12)), base),
            ((xi, xi * (e1 - e12)), (xi * (1 - e123), xi * (e1 - e123)), base),
        ]
    elif adjacency == "edge_adjacent":
        base = w * xi**3 * e1**2
        regions = [
            ((xi, xi * e1 * e3), (xi * (1 - e12), xi * e1 * (1 - e2)), base),
            ((xi, xi * e1), (xi * (1 - e123), xi * e12 * (1 - e3)), base * e2),
            ((xi * (1 - e12), xi * e1 * (1 - e2)), (xi, xi * e123), base * e2),
            ((xi * (1 - e123), xi * e12 * (1 - e3)), (xi, xi * e1), base * e2),
            ((xi * (1 - e123), xi * e1 * (1 - e2 * e3)), (xi, xi * e12), base * e2),
        ]
    elif adjacency == "vertex_adjacent":
        base = w * xi**3 * e2
        regions = [
            ((xi, xi * e1), (xi * e2, xi * e2 * e3), base),
            ((xi * e2, xi * e2 * e3), (xi, xi * e1), base),
        ]
    else:
        raise ValueError("Unknown adjacency.")
    del one
    # interleave regions per tensor point, as the reference enumerates them
    nr = len(regions)
    npts = nr * len(xi)
    test = _np.empty((2, npts))
    trial = _np.empty((2, npts))
    weights = _np.empty(npts)
    for r, ((ta, tb), (sa, sb), wr) in enumerate(regions):
        test[0, r::nr] = ta - tb
        test[1, r::nr] = tb
        trial[0, r::nr] = sa - sb
        trial[1, r::nr] = sb
        weights[r::nr] = wr
    return _np.asfortranarray(test), _np.asfortranarray(trial), weights


def remap_shared_vertex(points, vertex_id):
    """Move the shared vertex of a vertex-adjacent rule from 0 to ``vertex_id``."""
    if vertex_id == 0:
        return points.copy()
    out = _np.empty_like(points)
    if vertex_id == 1:
        out[0] = 1.0 - points[0] - points[1]
        out[1] = points[1]
    elif vertex_id == 2:
        out[0] = points[0]
        out[1] = 1.0 - points[0] - points[1]
    else:
        raise ValueError("vertex_id must be 0, 1 or 2")
    return out


_REF_VERTICES = _np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def remap_shared_edge(points, v0, v1):
    """Move the shared edge of an edge-adjacent rule from (0, 1) to (v0, v1).

    The affine map sends reference vertices 0, 1, 2 to vertices v0, v1 and
    the remaining one (duffy_galerkin.py:253-285).
    """
    nv = _REF_VERTICES[:, [v0, v1, 3 - v0 - v1]]
    a = _np.column_stack([nv[:, 1] - nv[:, 0], nv[:, 2] - nv[:, 0]])
    return _np.asfortranarray(a @ points + nv[:, :1])


# Ordering of the six edge remaps and the 3x3 lookup from (v0, v1) to that
# position (singular_assembler.py:281-344).
EDGE_REMAPS = [(0, 1), (1, 0), (1, 2), (2, 1), (0, 2), (2, 0)]
EDGE_REMAP_INDEX = _np.array([[-1, 0, 4], [1, -1, 2], [5, 3, -1]], dtype=_np.int64)


class SingularPairs(object):
    """Flattened singular pair list of a grid restricted to test/trial support.

    ``arrays()`` returns, in order: test_points (2, P), trial_points (2, P),
    weights (W,), test_elements, trial_elements, test_offsets, trial_offsets,
    weights_offsets, number_of_quad_points (all (npairs,) uint32).  Pairs are
    ordered coincident, then edge-adjacent, then vertex-adjacent.  The point
    table concatenates the coincident rule, the six edge remaps and the three
    vertex remaps; the weight table concatenates the three base rules.
    """

    def __init__(self, grid, order, test_support, trial_support):
        test_support = _np.asarray(test_support, dtype=bool)
        trial_support = _np.asarray(trial_support, dtype=bool)
        self.order = order
        self.coincident = _np.flatnonzero(test_support & trial_support)
        ea = grid.edge_adjacency
        va = grid.vertex_adjacency
        self.edge = ea[:, test_support[ea[0]] & trial_support[ea[1]]]
        self.vertex = va[:, test_support[va[0]] & trial_support[va[1]]]
        self.counts = (len(self.coincident), self.edge.shape[1], self.vertex.shape[1])

    @property
    def number_of_pairs(self):
        return sum(self.counts)

    def arrays(self):
        q = self.order
        nc = number_of_duffy_points(q, "coincident")
        ne_ = number_of_duffy_points(q, "edge_adjacent")
        nv = number_of_duffy_points(q, "vertex_adjacent")
        ct, cs, cw = duffy_rule(q, "coincident")
        et, es, ew = duffy_rule(q, "edge_adjacent")
        vt, vs, vw = duffy_rule(q, "vertex_adjacent")
        test_points = _np.hstack(
            [ct]
            + [remap_shared_edge(et, a, b) for a, b in EDGE_REMAPS]
            + [remap_shared_vertex(vt, k) for k in range(3)]
        )
        trial_points = _np.hstack(
            [cs]
            + [remap_shared_edge(es, a, b) for a, b in EDGE_REMAPS]
            + [remap_shared_vertex(vs, k) for k in range(3)]
        )
        weights = _np.hstack([cw, ew, vw])
        n0, n1, n2 = self.counts
        test_elements = _np.concatenate([self.coincident, self.edge[0], self.vertex[0]]).astype(_np.uint32)
        trial_elements = _np.concatenate([self.coincident, self.edge[1], self.vertex[1]]).astype(_np.uint32)
        edge_off = nc + ne_ * EDGE_REMAP_INDEX
        vert_off = nc + 6 * ne_ + nv * _np.arange(3)
        test_offsets = _np.concatenate(
            [_np.zeros(n0, _np.int64), edge_off[self.edge[2], self.edge[3]], vert_off[self.vertex[2]]]
        ).astype(_np.uint32)
        trial_offsets = _np.concatenate(
            [_np.zeros(n0, _np.int64), edge_off[self.edge[4], self.edge[5]], vert_off[self.vertex[3]]]
        ).astype(_np.uint32)
        weights_offsets = _np.concatenate(
            [_np.zeros(n0, _np.int64), _np.full(n1, nc), _np.full(n2, nc + ne_)]
        ).astype(_np.uint32)
        npoints = _np.concatenate([_np.full(n0, nc), _np.full(n1, ne_), _np.full(n2, nv)]).astype(_np.uint32)
        return [
            _np.asfortranarray(test_points),
            _np.asfortranarray(trial_points),
            weights,
            test_elements,
            trial_elements,
            test_offsets,
            trial_offsets,
            weights_offsets,
            npoints,
        ]
