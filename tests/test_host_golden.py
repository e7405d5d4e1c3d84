"""Host bookkeeping (adjacency, dof maps, quadrature) against the reference's own arrays."""

import numpy as np
import pytest

from conftest import load_golden


def _as_set(cols):
    return set(map(tuple, np.asarray(cols).T.tolist()))


def test_adjacency_matches_reference(sphere_msh_grid):
    h = load_golden("host_sphere_msh.npz")
    assert _as_set(sphere_msh_grid.edge_adjacency) == _as_set(h["edge_adjacency"])
    assert _as_set(sphere_msh_grid.vertex_adjacency) == _as_set(h["vertex_adjacency"])
    assert np.array_equal(sphere_msh_grid.element_edges, h["element_edges"])


@pytest.mark.parametrize("kind,deg", [("DP", 0), ("DP", 1), ("P", 1), ("RWG", 0), ("SNC", 0)])
def test_dof_maps_match_reference(sphere_msh_grid, kind, deg):
    from bempp_cuda.space import function_space

    h = load_golden("host_sphere_msh.npz")
    s = function_space(sphere_msh_grid, kind, deg)
    key = "%s%d" % (kind, deg)
    assert np.array_equal(s.local2global, h[key + "__l2g"])
    assert np.array_equal(s.local_multipliers, h[key + "__mult"])
    assert np.array_equal(s.support, h[key + "__support"])


def test_singular_pairs_match_reference(sphere_msh_grid):
    from bempp_cuda.quadrature import SingularPairs

    h = load_golden("host_sphere_msh.npz")
    sup = np.ones(sphere_msh_grid.number_of_elements, dtype=bool)
    mine = SingularPairs(sphere_msh_grid, 4, sup, sup).arrays()
    for idx, name in enumerate(["test_points", "trial_points", "weights"]):
        ref = h["singular__" + name]
        assert mine[idx].shape == ref.shape
        assert np.max(np.abs(mine[idx] - ref)) < 1e-14
    names = ["test_elements", "trial_elements", "test_offsets", "trial_offsets", "weights_offsets",
             "number_of_quad_points"]
    m = set(zip(*[mine[3 + k].tolist() for k in range(6)]))
    r = set(zip(*[h["singular__" + n].tolist() for n in names]))
    assert m == r


def test_triangle_rule_matches_reference():
    from bempp_cuda.quadrature import triangle_rule

    h = load_golden("host_sphere_msh.npz")
    p, w = triangle_rule(4)
    rp, rw = h["triangle4_points"], h["triangle4_weights"]
    a = np.lexsort((p[1], p[0]))
    b = np.lexsort((rp[1], rp[0]))
    assert np.max(np.abs(p[:, a] - rp[:, b])) < 1e-14
    assert np.max(np.abs(w[a] - rw[b])) < 1e-14


def test_regular_sphere_counts():
    from bempp_cuda.shapes import sphere_arrays

    for level, ne, nv in [(0, 8, 6), (4, 2048, 1026), (5, 8192, 4098)]:
        v, e = sphere_arrays(level)
        assert e.shape == (3, ne) and v.shape == (3, nv)
        assert np.allclose(np.linalg.norm(v, axis=0), 1.0)


def test_grid_rejects_bad_input():
    from bempp_cuda.grid import Grid

    v = np.array([[0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0], [0.0, 0.0, 0.0, 1.0]])
    with pytest.raises(ValueError):
        Grid(v, np.array([[0], [1], [7]]))
    with pytest.raises(ValueError):
        Grid(v, np.array([[0], [1], [1]]))  # zero area
    bad = v.copy()
    bad[0, 0] = np.nan
    with pytest.raises(ValueError):
        Grid(bad, np.array([[0], [1], [2]]))
