"""Operator cases shared by the oracle and GPU parity tests."""

import numpy as np

# key -> (factory path under bempp_cuda.operators.boundary, domain space, dual space, parameter or None)
BOUNDARY = {
    "laplace_slp_p0_p0": ("laplace.single_layer", ("DP", 0), ("DP", 0), None),
    "laplace_slp_p1_p1": ("laplace.single_layer", ("P", 1), ("P", 1), None),
    "laplace_slp_dp1_dp1": ("laplace.single_layer", ("DP", 1), ("DP", 1), None),
    "laplace_slp_dp1_p0": ("laplace.single_layer", ("DP", 1), ("DP", 0), None),
    "laplace_slp_p0_dp1": ("laplace.single_layer", ("DP", 0), ("DP", 1), None),
    "laplace_dlp_p1_p1": ("laplace.double_layer", ("P", 1), ("P", 1), None),
    "laplace_adlp_p1_p1": ("laplace.adjoint_double_layer", ("P", 1), ("P", 1), None),
    "laplace_hyp_p1_p1": ("laplace.hypersingular", ("P", 1), ("P", 1), None),
    "helmholtz_slp_p0_p0": ("helmholtz.single_layer", ("DP", 0), ("DP", 0), 2.5),
    "helmholtz_slp_p1_p1": ("helmholtz.single_layer", ("P", 1), ("P", 1), 2.5),
    "helmholtz_slp_dp1_p0": ("helmholtz.single_layer", ("DP", 1), ("DP", 0), 2.5),
    "helmholtz_slp_p0_dp1": ("helmholtz.single_layer", ("DP", 0), ("DP", 1), 2.5),
    "helmholtz_dlp_p1_p1": ("helmholtz.double_layer", ("P", 1), ("P", 1), 2.5),
    "helmholtz_adlp_p1_p1": ("helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 2.5),
    "helmholtz_hyp_p1_p1": ("helmholtz.hypersingular", ("P", 1), ("P", 1), 2.5),
    "helmholtz_c_slp_p1_p1": ("helmholtz.single_layer", ("P", 1), ("P", 1), 2.5 + 1j),
    "helmholtz_c_dlp_p1_p1": ("helmholtz.double_layer", ("P", 1), ("P", 1), 2.5 + 1j),
    "helmholtz_c_adlp_p1_p1": ("helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 2.5 + 1j),
    "helmholtz_c_hyp_p1_p1": ("helmholtz.hypersingular", ("P", 1), ("P", 1), 2.5 + 1j),
    "maxwell_efie_rwg_snc": ("maxwell.electric_field", ("RWG", 0), ("SNC", 0), 2.5),
    "maxwell_mfie_rwg_snc": ("maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), 2.5),
    "maxwell_c_efie_rwg_snc": ("maxwell.electric_field", ("RWG", 0), ("SNC", 0), 2.5 + 1j),
    "maxwell_c_mfie_rwg_snc": ("maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), 2.5 + 1j),
    "modhelm_slp_p0_p0": ("modified_helmholtz.single_layer", ("DP", 0), ("DP", 0), 1.5),
    "modhelm_dlp_p1_p1": ("modified_helmholtz.double_layer", ("P", 1), ("P", 1), 1.5),
    "modhelm_adlp_p1_p1": ("modified_helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 1.5),
    "modhelm_hyp_p1_p1": ("modified_helmholtz.hypersingular", ("P", 1), ("P", 1), 1.5),
    "helmholtz_dlp_p0_p0": ("helmholtz.double_layer", ("DP", 0), ("DP", 0), 5.0),
    "helmholtz_adlp_p0_p0": ("helmholtz.adjoint_double_layer", ("DP", 0), ("DP", 0), 5.0),
    "laplace_dlp_p0_p0": ("laplace.double_layer", ("DP", 0), ("DP", 0), None),
}

# key -> (factory path under bempp_cuda.operators, space, parameter or None)
POTENTIAL = {
    "laplace_slp_pot_p0": ("potential.laplace.single_layer", ("DP", 0), None),
    "laplace_slp_pot_p1": ("potential.laplace.single_layer", ("P", 1), None),
    "laplace_dlp_pot_p1": ("potential.laplace.double_layer", ("P", 1), None),
    "helmholtz_slp_pot_p1": ("potential.helmholtz.single_layer", ("P", 1), 2.5),
    "helmholtz_dlp_pot_p1": ("potential.helmholtz.double_layer", ("P", 1), 2.5),
    "helmholtz_c_slp_pot_p1": ("potential.helmholtz.single_layer", ("P", 1), 2.5 + 1j),
    "helmholtz_c_dlp_pot_p1": ("potential.helmholtz.double_layer", ("P", 1), 2.5 + 1j),
    "helmholtz_slp_ff_p1": ("far_field.helmholtz.single_layer", ("P", 1), 2.5),
    "helmholtz_dlp_ff_p1": ("far_field.helmholtz.double_layer", ("P", 1), 2.5),
    "maxwell_efield_pot": ("potential.maxwell.electric_field", ("RWG", 0), 2.5),
    "maxwell_mfield_pot": ("potential.maxwell.magnetic_field", ("RWG", 0), 2.5),
    "maxwell_c_efield_pot": ("potential.maxwell.electric_field", ("RWG", 0), 2.5 + 1j),
    "maxwell_c_mfield_pot": ("potential.maxwell.magnetic_field", ("RWG", 0), 2.5 + 1j),
    "maxwell_efield_ff": ("far_field.maxwell.electric_field", ("RWG", 0), 2.5),
    "maxwell_mfield_ff": ("far_field.maxwell.magnetic_field", ("RWG", 0), 2.5),
}


def resolve(path):
    from bempp_cuda import operators

    obj = operators
    for part in path.split("."):
        obj = getattr(obj, part)
    return obj


def boundary_operator(key, grid):
    """Build (operator, domain, dual) for a boundary case on ``grid`` with bempp_cuda objects."""
    from bempp_cuda.space import function_space

    path, dsp, tsp, k = BOUNDARY[key]
    domain = function_space(grid, *dsp)
    dual = function_space(grid, *tsp)
    factory = resolve("boundary." + path)
    op = factory(domain, domain, dual) if k is None else factory(domain, domain, dual, k)
    return op, domain, dual


def oracle_dense(orc, op, domain, dual):
    """Oracle weak form of ``op`` (same host inputs as the product)."""
    from bempp_cuda.quadrature import SingularPairs, triangle_rule

    d = op.descriptor
    qp, qw = triangle_rule(op.parameters.quadrature.regular)
    rule = None
    if domain.grid == dual.grid:
        rule = SingularPairs(domain.grid, op.parameters.quadrature.singular, dual.support, domain.support).arrays()
    return orc.assemble_dense(d.kernel_type, d.assembly_type, d.options, d.is_complex, domain, dual, qp, qw, rule)


def potential_operator(key, grid, points):
    from bempp_cuda.space import function_space

    path, sp, k = POTENTIAL[key]
    space = function_space(grid, *sp)
    factory = resolve(path)
    op = factory(space, points) if k is None else factory(space, points, k)
    return op, space


def oracle_potential(orc, op, space, coefficients):
    from bempp_cuda.quadrature import triangle_rule

    d = op.descriptor
    qp, qw = triangle_rule(op.parameters.quadrature.regular)
    return orc.evaluate_potential(d.kernel_type, d.assembly_type, d.options, space, op.points, coefficients, qp, qw)


def sphere_shell_points(n, seed):
    rng = np.random.default_rng(seed)
    dirs = rng.standard_normal((3, n))
    dirs /= np.linalg.norm(dirs, axis=0)
    radius = (1.5**3 + rng.random(n) * (3.0**3 - 1.5**3)) ** (1.0 / 3.0)
    return dirs * radius, dirs
