"""Mesh generators and a gmsh 2.2 reader.

``regular_sphere(level)`` replaces ``bempp_cl.api.shapes.regular_sphere``
(bempp_cl/api/shapes/shapes.py:114-138), whose data file is not shipped with
the reference.  It subdivides an octahedron ``level`` times, splitting every
triangle into four and projecting new vertices onto the unit sphere, which
gives 8 * 4**level outward-oriented triangles and 4 * 4**level + 2 vertices
(L4: 2048 / 1026, L5: 8192 / 4098, L6: 32768 / 16386).
"""

import functools as _functools

import numpy as _np

from .grid import Grid


def _octahedron():
    vertices = _np.array(
        [[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], dtype=_np.float64
    )
    faces = _np.array(
        [[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5], [0, 3, 5]], dtype=_np.int64
    )
    return vertices, faces


@_functools.lru_cache(maxsize=16)
def _sphere_arrays_cached(level):
    vertices, faces = _octahedron()
    verts = vertices.copy()
    for _ in range(level):
        nv = verts.shape[0]
        # the three edges of every face, as sorted vertex pairs
        e = _np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        key = _np.minimum(e[:, 0], e[:, 1]) * nv + _np.maximum(e[:, 0], e[:, 1])
        uniq, inverse = _np.unique(key, return_inverse=True)
        # number new vertices by first appearance (face-major, edge ab, bc, ca)
        nf = faces.shape[0]
        idx = _np.arange(3 * nf)
        order_key = _np.full(len(uniq), 3 * nf, dtype=_np.int64)
        _np.minimum.at(order_key, inverse, (idx % nf) * 3 + idx // nf)
        rank = _np.empty(len(uniq), dtype=_np.int64)
        rank[_np.argsort(order_key, kind="stable")] = _np.arange(len(uniq))
        lo = uniq // nv
        hi = uniq % nv
        mids = verts[lo] + verts[hi]
        mids /= _np.linalg.norm(mids, axis=1, keepdims=True)
        new_verts = _np.empty((nv + len(uniq), 3))
        new_verts[:nv] = verts
        new_verts[nv + rank] = mids
        m = nv + rank[inverse]
        ab, bc, ca = m[:nf], m[nf : 2 * nf], m[2 * nf :]
        a_, b_, c_ = faces[:, 0], faces[:, 1], faces[:, 2]
        new_faces = _np.empty((4 * nf, 3), dtype=_np.int64)
        new_faces[0::4] = _np.stack([a_, ab, ca], axis=1)
        new_faces[1::4] = _np.stack([ab, b_, bc], axis=1)
        new_faces[2::4] = _np.stack([ca, bc, c_], axis=1)
        new_faces[3::4] = _np.stack([ab, bc, ca], axis=1)
        verts, faces = new_verts, new_faces
    return verts.T.copy(), faces.T.copy()


def sphere_arrays(level):
    """Return (vertices (3, nv), elements (3, ne)) of the subdivided octahedron."""
    if level < 0:
        raise ValueError("level must be non-negative")
    v, e = _sphere_arrays_cached(int(level))
    return v.copy(), e.copy()


def regular_sphere(level):
    """Unit sphere grid with 8 * 4**level triangles."""
    v, e = sphere_arrays(level)
    return Grid(v, e)


def ellipsoid(level, r1=1.0, r2=1.0, r3=1.0, origin=(0.0, 0.0, 0.0)):
    """Sphere of ``level`` scaled per axis by (r1, r2, r3) and shifted."""
    v, e = sphere_arrays(level)
    v = v * _np.array([[r1], [r2], [r3]]) + _np.asarray(origin, dtype=_np.float64).reshape(3, 1)
    return Grid(v, e)


def real_spherical_harmonics(lmax, theta, phi):
    """Real spherical harmonics Y_lm (l <= lmax) at polar angle theta, azimuth phi.

    Returns an array (nharm, npoints) ordered l = 0..lmax, m = -l..l, with
    orthonormal scaling on the unit sphere.
    """
    from scipy.special import sph_harm_y

    out = []
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            y = sph_harm_y(l, abs(m), theta, phi)
            if m < 0:
                out.append(_np.sqrt(2.0) * (-1) ** m * y.imag)
            elif m == 0:
                out.append(y.real)
            else:
                out.append(_np.sqrt(2.0) * (-1) ** m * y.real)
    return _np.array(out)


def perturbed_sphere(level, lmax=4, sigma=0.02, seed=0):
    """Unit sphere with radius r = 1 + sum_lm a_lm Y_lm, a_lm ~ N(0, sigma^2)."""
    v, e = sphere_arrays(level)
    rng = _np.random.default_rng(seed)
    theta = _np.arccos(_np.clip(v[2], -1.0, 1.0))
    phi = _np.arctan2(v[1], v[0])
    ylm = real_spherical_harmonics(lmax, theta, phi)
    coeffs = rng.normal(0.0, sigma, size=ylm.shape[0])
    radius = 1.0 + coeffs @ ylm
    return Grid(v * radius, e), coeffs


def read_gmsh(path):
    """Read triangles and nodes of a gmsh 2.2 file (ASCII or binary).

    Returns (vertices (3, nv), elements (3, ne), physical tags (ne,)).  Only
    3-node triangles (type 2) are kept; node ids are renumbered densely.
    """
    import struct

    with open(path, "rb") as handle:
        data = handle.read()

    def section(name):
        start = data.index(b"$" + name + b"\n") + len(name) + 2
        end = data.index(b"$End" + name, start)
        return data[start:end]

    header = section(b"MeshFormat").split(b"\n")[0].split()
    binary = header[1] == b"1"
    nodes_raw = section(b"Nodes")
    elems_raw = section(b"Elements")
    node_ids = {}
    coords = []
    if binary:
        nl = nodes_raw.index(b"\n")
        nnodes = int(nodes_raw[:nl])
        body = nodes_raw[nl + 1 :]
        for k in range(nnodes):
            nid, x, y, z = struct.unpack_from("<iddd", body, 28 * k)
            node_ids[nid] = k
            coords.append((x, y, z))
        nl = elems_raw.index(b"\n")
        nelem = int(elems_raw[:nl])
        body = elems_raw[nl + 1 :]
        pos = 0
        tris, tags = [], []
        read = 0
        while read < nelem:
            etype, count, ntags = struct.unpack_from("<iii", body, pos)
            pos += 12
            nnode = {1: 2, 2: 3, 3: 4, 4: 4, 15: 1}[etype]
            for _ in range(count):
                vals = struct.unpack_from("<%di" % (1 + ntags + nnode), body, pos)
                pos += 4 * (1 + ntags + nnode)
                if etype == 2:
                    tris.append([node_ids[n] for n in vals[1 + ntags :]])
                    tags.append(vals[1] if ntags else 0)
            read += count
    else:
        lines = nodes_raw.decode().split("\n")
        nnodes = int(lines[0])
        for k in range(nnodes):
            parts = lines[1 + k].split()
            node_ids[int(parts[0])] = k
            coords.append(tuple(float(p) for p in parts[1:4]))
        lines = elems_raw.decode().split("\n")
        nelem = int(lines[0])
        tris, tags = [], []
        for k in range(nelem):
            parts = [int(p) for p in lines[1 + k].split()]
            if parts[1] == 2:
                ntags = parts[2]
                tris.append([node_ids[n] for n in parts[3 + ntags :]])
                tags.append(parts[3] if ntags else 0)
    vertices = _np.array(coords, dtype=_np.float64).T.copy()
    elements = _np.array(tris, dtype=_np.uint32).T.copy()
    return vertices, elements, _np.array(tags, dtype=_np.uint32)
