"""The numpy oracle restated from the reference, pinned to the reference's own
outputs (golden fixtures produced by the compiled reference)."""
import numpy as np
import pytest

import golden_cases as gc
from oracle import dfr_numpy

CASES = gc.names()


def test_fixtures_present():
    assert len(CASES) >= 10


@pytest.mark.parametrize("name", CASES)
def test_oracle_residual_matches_reference(name):
    g = gc.load(name)
    R = dfr_numpy.residual(g.setup(), g.U0, g.params, g.viscous)
    # same arithmetic as the reference up to summation order (and, on triangles,
    # the dense 'M3' operators' rounding): 1e-12 per variable scale
    assert gc.rel_err(R, g.R0) < 1e-12


@pytest.mark.parametrize("name", [n for n in CASES if gc.load(n).meta["nsteps"] <= 2])
def test_oracle_rk44_matches_reference(name):
    g = gc.load(name)
    st = g.setup()
    U = g.U0
    for _ in range(g.meta["nsteps"]):
        U = dfr_numpy.rk44_step(st, U, g.params, g.viscous, g.meta["dt"])
    assert gc.rel_err(U, g.Un) < 1e-12


def test_oracle_detects_planted_error():
    """A deliberately wrong oracle (flux sign flipped on one variable) must fail the check."""
    g = gc.load("quad_p3_euler_vortex")
    st = g.setup()
    bad = dfr_numpy.Setup(**{**st.__dict__, "oppDiv_fpts": st.oppDiv_fpts * 1.000001})
    R = dfr_numpy.residual(bad, g.U0, g.params, g.viscous)
    assert gc.rel_err(R, g.R0) > 1e-9
