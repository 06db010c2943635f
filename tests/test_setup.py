"""Host set-up of libzefr_b200 (no GPU): operators, metrics and face connectivity
must equal the reference's arrays exactly."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200.solver import Plan, make_params

CASES = gc.names()
EXACT = ["oppE", "oppD", "oppD_fpts", "oppDiv", "oppDiv_fpts", "coord_spts", "jaco_det_spts", "inv_jaco_spts",
         "fpt_partner", "fpt_slot", "fpt_norm", "fpt_dA"]


@pytest.mark.parametrize("name", CASES)
def test_setup_bit_exact(name):
    g = gc.load(name)
    plan = Plan(g.mesh, make_params(g.order, g.viscous), g.bounds)
    for key in EXACT:
        a = plan.get(key)
        b = g.setup_arrays[key]
        assert a.shape == b.shape, key
        if name.startswith("tri_") and key not in ("fpt_partner", "fpt_slot"):
            # triangles: the Vandermonde inverse and the orthonormal basis are
            # computed independently of the reference's (Eigen inverse, HiFiLES
            # Jacobi recurrence); same operators up to rounding
            assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max()), \
                f"{key}: max diff {np.abs(a - b).max()}"
        elif g.order <= 4 or key in ("fpt_partner", "fpt_slot"):
            # closed-form Gauss-Legendre nodes (P <= 4): identical doubles
            assert np.array_equal(a, b), f"{key}: max diff {np.abs(a - b).max()}"
        else:
            # P >= 5: the reference uses 15-digit node tables; operators agree to a few ulp
            assert np.abs(a - b).max() <= 1e-14 * max(1.0, np.abs(b).max()), key


def test_plan_info_counts():
    g = gc.load("hex_p3_ns_tgv")
    plan = Plan(g.mesh, make_params(3, True), g.bounds)
    info = plan.info
    assert (info.nspts, info.nfpts, info.nvars, info.ndims) == (64, 96, 5, 3)
    assert info.n_eles == 27 and info.n_gfpts_bnd == 0
    assert info.n_gfpts_int == 27 * 3 * 16
