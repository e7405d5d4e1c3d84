"""Generate the committed golden fixtures under tests/golden/.

Run once in a container where the reference bempp-cl source tree is present:

    PYTHONDONTWRITEBYTECODE=1 NUMBA_CACHE_DIR=/tmp/numba_cache \
        python tests/golden/make_golden.py /path/to/bempp-cl

It imports the reference from that path (with a stub for the absent meshio
module) and writes small .npz files:

* ``sphere_msh.npz``        mesh of test/data/sphere.msh (117 vertices, 230
                            triangles) read with bempp_cuda.shapes.read_gmsh
* ``legacy_boundary.npz``   fingerprints of the reference's own golden matrices
                            test/data/*_boundary*.npy: y = A u, z = A^T w for the
                            seeded complex vectors of ``probe_vectors``, ||A||_F
                            and 48 sampled entries
* ``legacy_potential.npz``  the reference's golden potential / far-field files
                            (points, coefficient vector, result)
* ``numba_boundary.npz``    full matrices from the reference Numba path on
                            regular_sphere(1) (32 triangles) for every operator
* ``numba_potential.npz``   reference Numba potentials on regular_sphere(2)
* ``host_sphere_msh.npz``   reference host bookkeeping on sphere.msh: edge and
                            vertex adjacency, dof maps of every space, singular
                            pair arrays at order 4 and the order-4 triangle rule
* ``identity.npz``          sparse L2 identities: the reference's golden
                            test/data/sparse_identity_*.npy on sphere.msh and
                            the live reference Numba path on regular_sphere(2)
                            for more space pairs, as nonzero triplets
                            (``--identity`` writes only this file)

Nothing at test time reads the reference tree; only these fixtures.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

BOUNDARY_CASES = [
    # (key, module.function, domain space, dual space, wavenumber, legacy file or None)
    ("laplace_slp_p0_p0", "laplace.single_layer", ("DP", 0), ("DP", 0), None, "laplace_single_layer_boundary_p0_p0"),
    ("laplace_slp_p1_p1", "laplace.single_layer", ("P", 1), ("P", 1), None, "laplace_single_layer_boundary_p1_p1"),
    ("laplace_slp_dp1_dp1", "laplace.single_layer", ("DP", 1), ("DP", 1), None, "laplace_single_layer_boundary_dp1_dp1"),
    ("laplace_slp_dp1_p0", "laplace.single_layer", ("DP", 1), ("DP", 0), None, "laplace_single_layer_boundary_p0_dp1"),
    ("laplace_slp_p0_dp1", "laplace.single_layer", ("DP", 0), ("DP", 1), None, "laplace_single_layer_boundary_dp1_p0"),
    ("laplace_dlp_p1_p1", "laplace.double_layer", ("P", 1), ("P", 1), None, "laplace_double_layer_boundary"),
    ("laplace_adlp_p1_p1", "laplace.adjoint_double_layer", ("P", 1), ("P", 1), None, "laplace_adj_double_layer_boundary"),
    ("laplace_hyp_p1_p1", "laplace.hypersingular", ("P", 1), ("P", 1), None, "laplace_hypersingular_boundary"),
    ("helmholtz_slp_p0_p0", "helmholtz.single_layer", ("DP", 0), ("DP", 0), 2.5, "helmholtz_single_layer_boundary_p0_p0"),
    ("helmholtz_slp_p1_p1", "helmholtz.single_layer", ("P", 1), ("P", 1), 2.5, "helmholtz_single_layer_boundary_p1_p1"),
    ("helmholtz_slp_dp1_p0", "helmholtz.single_layer", ("DP", 1), ("DP", 0), 2.5, "helmholtz_single_layer_boundary_p0_dp1"),
    ("helmholtz_slp_p0_dp1", "helmholtz.single_layer", ("DP", 0), ("DP", 1), 2.5, "helmholtz_single_layer_boundary_dp1_p0"),
    ("helmholtz_dlp_p1_p1", "helmholtz.double_layer", ("P", 1), ("P", 1), 2.5, "helmholtz_double_layer_boundary"),
    ("helmholtz_adlp_p1_p1", "helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 2.5, "helmholtz_adj_double_layer_boundary"),
    ("helmholtz_hyp_p1_p1", "helmholtz.hypersingular", ("P", 1), ("P", 1), 2.5, "helmholtz_hypersingular_boundary"),
    ("helmholtz_c_slp_p1_p1", "helmholtz.single_layer", ("P", 1), ("P", 1), 2.5 + 1j, "helmholtz_complex_single_layer_boundary"),
    ("helmholtz_c_dlp_p1_p1", "helmholtz.double_layer", ("P", 1), ("P", 1), 2.5 + 1j, "helmholtz_complex_double_layer_boundary"),
    ("helmholtz_c_adlp_p1_p1", "helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 2.5 + 1j, "helmholtz_complex_adj_double_layer_boundary"),
    ("helmholtz_c_hyp_p1_p1", "helmholtz.hypersingular", ("P", 1), ("P", 1), 2.5 + 1j, "helmholtz_complex_hypersingular_boundary"),
    ("maxwell_efie_rwg_snc", "maxwell.electric_field", ("RWG", 0), ("SNC", 0), 2.5, "maxwell_electric_field_boundary"),
    ("maxwell_mfie_rwg_snc", "maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), 2.5, "maxwell_magnetic_field_boundary"),
    ("maxwell_c_efie_rwg_snc", "maxwell.electric_field", ("RWG", 0), ("SNC", 0), 2.5 + 1j, "maxwell_electric_field_complex_boundary"),
    ("maxwell_c_mfie_rwg_snc", "maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), 2.5 + 1j, "maxwell_magnetic_field_complex_boundary"),
    ("modhelm_slp_p0_p0", "modified_helmholtz.single_layer", ("DP", 0), ("DP", 0), 1.5, None),
    ("modhelm_dlp_p1_p1", "modified_helmholtz.double_layer", ("P", 1), ("P", 1), 1.5, None),
    ("modhelm_adlp_p1_p1", "modified_helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 1.5, None),
    ("modhelm_hyp_p1_p1", "modified_helmholtz.hypersingular", ("P", 1), ("P", 1), 1.5, None),
    ("helmholtz_dlp_p0_p0", "helmholtz.double_layer", ("DP", 0), ("DP", 0), 5.0, None),
    ("helmholtz_adlp_p0_p0", "helmholtz.adjoint_double_layer", ("DP", 0), ("DP", 0), 5.0, None),
    ("laplace_dlp_p0_p0", "laplace.double_layer", ("DP", 0), ("DP", 0), None, None),
]

POTENTIAL_LEGACY = [
    # (key, module.function, space, wavenumber, legacy file)
    ("laplace_slp_pot_p0", "potential.laplace.single_layer", ("DP", 0), None, "laplace_single_layer_potential_p0"),
    ("laplace_slp_pot_p1", "potential.laplace.single_layer", ("P", 1), None, "laplace_single_layer_potential_p1"),
    ("laplace_dlp_pot_p1", "potential.laplace.double_layer", ("P", 1), None, "laplace_double_layer_potential_p1"),
    ("helmholtz_slp_pot_p1", "potential.helmholtz.single_layer", ("P", 1), 2.5, "helmholtz_single_layer_potential_p1"),
    ("helmholtz_dlp_pot_p1", "potential.helmholtz.double_layer", ("P", 1), 2.5, "helmholtz_double_layer_potential_p1"),
    ("helmholtz_c_slp_pot_p1", "potential.helmholtz.single_layer", ("P", 1), 2.5 + 1j, "helmholtz_single_layer_potential_complex_p1"),
    ("helmholtz_c_dlp_pot_p1", "potential.helmholtz.double_layer", ("P", 1), 2.5 + 1j, "helmholtz_double_layer_potential_complex_p1"),
    ("helmholtz_slp_ff_p1", "far_field.helmholtz.single_layer", ("P", 1), 2.5, "helmholtz_single_layer_far_field_p1"),
    ("helmholtz_dlp_ff_p1", "far_field.helmholtz.double_layer", ("P", 1), 2.5, "helmholtz_double_layer_far_field_p1"),
    ("maxwell_efield_pot", "potential.maxwell.electric_field", ("RWG", 0), 2.5, "maxwell_electric_field_potential"),
    ("maxwell_mfield_pot", "potential.maxwell.magnetic_field", ("RWG", 0), 2.5, "maxwell_magnetic_field_potential"),
    ("maxwell_c_efield_pot", "potential.maxwell.electric_field", ("RWG", 0), 2.5 + 1j, "maxwell_electric_field_potential_complex"),
    ("maxwell_c_mfield_pot", "potential.maxwell.magnetic_field", ("RWG", 0), 2.5 + 1j, "maxwell_magnetic_field_potential_complex"),
    ("maxwell_efield_ff", "far_field.maxwell.electric_field", ("RWG", 0), 2.5, "maxwell_electric_far_field"),
    ("maxwell_mfield_ff", "far_field.maxwell.magnetic_field", ("RWG", 0), 2.5, "maxwell_magnetic_far_field"),
]


def probe_vectors(rows, cols, seed=1234):
    """Seeded complex probe vectors u (cols, 2) and w (rows, 2) and 48 entry indices."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((cols, 2)) + 1j * rng.standard_normal((cols, 2))
    w = rng.standard_normal((rows, 2)) + 1j * rng.standard_normal((rows, 2))
    ii = rng.integers(0, rows, 48)
    jj = rng.integers(0, cols, 48)
    return u, w, ii, jj


def fingerprint(mat, seed=1234):
    """Seeded projections of a matrix that pin every entry to ~1e-15 relative."""
    rows, cols = mat.shape
    u, w, ii, jj = probe_vectors(rows, cols, seed)
    return {
        "Au": mat @ u,
        "ATw": mat.T @ w,
        "fro": np.array(np.linalg.norm(mat)),
        "entries": mat[ii, jj],
        "shape": np.array(mat.shape),
    }


# (key, domain space, dual space, legacy file or None); the identity's range is its domain
IDENTITY_CASES = [
    ("p0_p0", ("DP", 0), ("DP", 0), "sparse_identity_p0_p0"),
    ("p1_p1", ("P", 1), ("P", 1), "sparse_identity_p1_p1"),
    ("p0_p1", ("P", 1), ("DP", 0), "sparse_identity_p0_p1"),
    ("p1_p0", ("DP", 0), ("P", 1), "sparse_identity_p1_p0"),
    ("snc_rwg", ("RWG", 0), ("SNC", 0), "sparse_identity_snc_rwg"),
    ("dp1_dp1", ("DP", 1), ("DP", 1), None),
    ("p1_dp1", ("DP", 1), ("P", 1), None),
    ("rwg_rwg", ("RWG", 0), ("RWG", 0), None),
    ("snc_snc", ("SNC", 0), ("SNC", 0), None),
    ("rwg_snc", ("SNC", 0), ("RWG", 0), None),
]


def _triplets(mat):
    mat = np.asarray(mat)
    r, c = np.nonzero(mat)
    return r.astype(np.int32), c.astype(np.int32), mat[r, c], np.array(mat.shape)


def make_identity(ref_root):
    sys.modules.setdefault("meshio", types.ModuleType("meshio"))
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(REPO, "bempp-cl_b200"))
    import bempp_cl.api as api
    from bempp_cl.api.grid.grid import Grid as RefGrid
    from bempp_cl.api.operators.boundary.sparse import identity
    from bempp_cuda import shapes

    api.GLOBAL_PARAMETERS.quadrature.regular = 4
    data = os.path.join(ref_root, "test", "data")
    out = {}
    for key, dsp, tsp, gold in IDENTITY_CASES:
        if gold is None:
            continue
        for name, val in zip(("rows", "cols", "vals", "shape"), _triplets(np.load(os.path.join(data, gold + ".npy")))):
            out["legacy_%s__%s" % (key, name)] = val
    sv, se = shapes.sphere_arrays(2)
    g = RefGrid(sv, se)
    out["vertices"], out["elements"] = sv, se
    for key, dsp, tsp, gold in IDENTITY_CASES:
        d = api.function_space(g, *dsp)
        t = api.function_space(g, *tsp)
        mat = identity(d, d, t, device_interface="numba").weak_form().to_dense()
        for name, val in zip(("rows", "cols", "vals", "shape"), _triplets(mat)):
            out["live_%s__%s" % (key, name)] = val
        out["live_%s__spaces" % key] = np.array([dsp[0], str(dsp[1]), tsp[0], str(tsp[1])])
    np.savez_compressed(os.path.join(HERE, "identity.npz"), **out)
    print("identity fixtures written to", HERE)


def main(ref_root):
    sys.modules.setdefault("meshio", types.ModuleType("meshio"))
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(REPO, "bempp-cl_b200"))
    import bempp_cl.api as api
    from bempp_cl.api.grid.grid import Grid as RefGrid
    from bempp_cl.api.integration import triangle_gauss
    from bempp_cl.core.singular_assembler import _SingularQuadratureRuleInterfaceGalerkin
    from bempp_cuda import shapes

    data = os.path.join(ref_root, "test", "data")
    params = api.GLOBAL_PARAMETERS
    params.quadrature.regular = 4
    params.quadrature.singular = 4

    v, e, tags = shapes.read_gmsh(os.path.join(data, "sphere.msh"))
    np.savez_compressed(os.path.join(HERE, "sphere_msh.npz"), vertices=v, elements=e, tags=tags)
    grid = RefGrid(v, e)

    def resolve(path):
        obj = api.operators
        for part in path.split("."):
            obj = getattr(obj, part)
        return obj

    def boundary_op(name, dsp, tsp, k, g):
        f = resolve("boundary." + name)
        d = api.function_space(g, *dsp)
        t = api.function_space(g, *tsp)
        args = (d, d, t) if k is None else (d, d, t, k)
        return f(*args, assembler="dense", device_interface="numba")

    # legacy golden matrices -> fingerprints
    legacy = {}
    for key, name, dsp, tsp, k, gold in BOUNDARY_CASES:
        if gold is None:
            continue
        mat = np.load(os.path.join(data, gold + ".npy"))
        for fk, fv in fingerprint(mat).items():
            legacy[key + "__" + fk] = fv
        legacy[key + "__spaces"] = np.array([dsp[0], str(dsp[1]), tsp[0], str(tsp[1])])
        legacy[key + "__k"] = np.array(complex(k) if k is not None else np.nan + 0j)
        legacy[key + "__op"] = np.array(name)
    np.savez_compressed(os.path.join(HERE, "legacy_boundary.npz"), **legacy)

    # legacy golden potentials (small: 10 points)
    pots = {}
    for key, name, sp, k, gold in POTENTIAL_LEGACY:
        d = np.load(os.path.join(data, gold + ".npz"))
        pots[key + "__points"] = d["points"]
        pots[key + "__vec"] = d["vec"]
        pots[key + "__result"] = d["result"]
        pots[key + "__space"] = np.array([sp[0], str(sp[1])])
        pots[key + "__k"] = np.array(complex(k) if k is not None else np.nan + 0j)
        pots[key + "__op"] = np.array(name)
    np.savez_compressed(os.path.join(HERE, "legacy_potential.npz"), **pots)

    # live reference Numba matrices on regular_sphere(1)
    sv, se = shapes.sphere_arrays(1)
    small = RefGrid(sv, se)
    live = {"vertices": sv, "elements": se}
    for key, name, dsp, tsp, k, gold in BOUNDARY_CASES:
        op = boundary_op(name, dsp, tsp, k, small)
        live[key + "__A"] = op.weak_form().A
        desc = op.descriptor
        live[key + "__desc"] = np.array([desc.kernel_type, desc.assembly_type])
        live[key + "__options"] = np.array(desc.options, dtype=np.float64)
        live[key + "__spaces"] = np.array([dsp[0], str(dsp[1]), tsp[0], str(tsp[1])])
    np.savez_compressed(os.path.join(HERE, "numba_boundary.npz"), **live)

    # live reference Numba potentials on regular_sphere(2), seeded shell points
    pv, pe = shapes.sphere_arrays(2)
    pgrid = RefGrid(pv, pe)
    rng = np.random.default_rng(7)
    npts = 40
    dirs = rng.standard_normal((3, npts))
    dirs /= np.linalg.norm(dirs, axis=0)
    radius = (1.5**3 + rng.random(npts) * (3.0**3 - 1.5**3)) ** (1.0 / 3.0)
    points = dirs * radius
    livep = {"vertices": pv, "elements": pe, "points": points, "directions": dirs}
    for key, name, sp, k, gold in POTENTIAL_LEGACY:
        space = api.function_space(pgrid, *sp)
        coeffs = rng.standard_normal(space.global_dof_count) + 1j * rng.standard_normal(space.global_dof_count)
        f = resolve(name)
        pts = dirs if "far_field" in name else points
        op = f(space, pts) if k is None else f(space, pts, k)
        from bempp_cl.api.assembly.grid_function import GridFunction

        res = op.evaluate(GridFunction(space, coefficients=coeffs))
        livep[key + "__coeffs"] = coeffs
        livep[key + "__result"] = res
    np.savez_compressed(os.path.join(HERE, "numba_potential.npz"), **livep)

    # reference host bookkeeping on sphere.msh
    host = {}
    host["edge_adjacency"] = grid.edge_adjacency
    host["vertex_adjacency"] = grid.vertex_adjacency
    host["element_edges"] = grid.element_edges
    for kind, deg in [("DP", 0), ("DP", 1), ("P", 1), ("RWG", 0), ("SNC", 0)]:
        s = api.function_space(grid, kind, deg)
        host["%s%d__l2g" % (kind, deg)] = s.local2global
        host["%s%d__mult" % (kind, deg)] = s.local_multipliers
        host["%s%d__support" % (kind, deg)] = s.support
    sup = np.ones(grid.number_of_elements, dtype=bool)
    arrays = _SingularQuadratureRuleInterfaceGalerkin(grid, 4, sup, sup).get_arrays()
    names = ["test_points", "trial_points", "weights", "test_elements", "trial_elements", "test_offsets",
             "trial_offsets", "weights_offsets", "number_of_quad_points"]
    for n, a in zip(names, arrays):
        host["singular__" + n] = np.asarray(a)
    qp, qw = triangle_gauss.rule(4)
    host["triangle4_points"] = qp
    host["triangle4_weights"] = qw
    np.savez_compressed(os.path.join(HERE, "host_sphere_msh.npz"), **host)
    make_identity(ref_root)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    argv = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not argv:
        sys.exit("usage: make_golden.py REFERENCE_CHECKOUT [--identity]")
    root = argv[0]
    if "--identity" in sys.argv[1:]:
        make_identity(root)
    else:
        main(root)
