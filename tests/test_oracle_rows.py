"""The oracle's row sample equals the rows of its full assembly (CPU).

The GPU parity tests at the configured sizes (regular_sphere(5) P1,
regular_sphere(4) RWG, regular_sphere(6) DP0) compare sampled rows only,
because the oracle cannot assemble those matrices whole in seconds; this pins
the sampling itself on a small grid, every space pairing of the cases.
"""

import numpy as np
import pytest

import cases


@pytest.mark.parametrize("key", ["helmholtz_slp_p1_p1", "helmholtz_hyp_p1_p1", "helmholtz_c_adlp_p1_p1",
                                 "maxwell_efie_rwg_snc", "maxwell_mfie_rwg_snc", "helmholtz_dlp_p0_p0",
                                 "laplace_slp_dp1_p0", "laplace_slp_p0_dp1"])
def test_row_sample_equals_full_rows(oracle, key):
    from bempp_cuda.quadrature import triangle_rule
    from bempp_cuda.shapes import regular_sphere

    grid = regular_sphere(1)
    op, domain, dual = cases.boundary_operator(key, grid)
    full = cases.oracle_dense(oracle, op, domain, dual)
    rows = np.sort(np.random.default_rng(3).choice(dual.global_dof_count, 9, replace=False))
    qp, qw = triangle_rule(4)
    d = op.descriptor
    got = oracle.assemble_rows(d.kernel_type, d.assembly_type, d.options, d.is_complex, domain, dual, rows, qp, qw)
    assert got.shape == (len(rows), domain.global_dof_count)
    np.testing.assert_allclose(got, full[rows], rtol=0, atol=1e-14 * np.abs(full).max())
