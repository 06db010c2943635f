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


@pytest.mark.parametrize("name", gc.diag_names())
def test_residual_norm_definition_matches_reference(name):
    """report_residuals prints max, sum of |.| and sqrt of the sum of squares of
    divF/|J| per variable divided by nSpts * nEles: the definition the
    library's zb_residual_norms implements, applied to the golden residual."""
    g, d = gc.load(name), gc.load_diag(name)
    S, V, E = g.R0.shape
    r = g.R0 / g.setup_arrays["jaco_det_spts"].reshape(S, 1, E)
    n = S * E
    assert np.allclose(np.abs(r).max(axis=(0, 2)) / n, d["res_max"], rtol=1e-14, atol=0)
    assert np.allclose(np.abs(r).sum(axis=(0, 2)) / n, d["res_l1"], rtol=1e-12, atol=0)
    assert np.allclose(np.sqrt((r * r).sum(axis=(0, 2))) / n, d["res_l2"], rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", [n for n in gc.diag_names() if "turb" in gc.load_diag(n)])
def test_oracle_functionals_match_reference(name):
    """The restated kinetic energy and enstrophy integrals, normalised as
    report_turbulent_stats prints them, against the reference's own output."""
    g, d = gc.load(name), gc.load_diag(name)
    from zefr_b200.solver import Plan, params_from_reference
    w = Plan(g.mesh, params_from_reference(g.params, g.order), g.bounds).get("weights_spts")
    fo = dfr_numpy.functionals(g.setup(), g.U0, w, g.params, g.viscous)
    ke, en, norm = d["turb"]
    assert abs(fo["ke"] / norm - ke) <= 1e-13 * abs(ke)
    assert abs(fo["enstrophy"] / norm - en) <= 1e-12 * abs(en)


@pytest.mark.parametrize("name", [n for n in gc.diag_names() if "force" in gc.load_diag(n)])
def test_oracle_wall_force_matches_reference(name):
    """The restated wall force and moment (2D) against the reference's own
    compute_moments on the same state."""
    g, d = gc.load(name), gc.load_diag(name)
    from zefr_b200.solver import Plan, params_from_reference
    plan = Plan(g.mesh, params_from_reference(g.params, g.order), g.bounds)
    st = g.setup()
    Fp = st.oppE.shape[0]
    N = g.order + 1
    w1 = np.polynomial.legendre.leggauss(N)[1]
    wf = np.array([w1[f % N] for f in range(Fp)])
    S, V, E = g.U0.shape
    cfp = plan.get("coord_fpts").reshape(Fp, g.meta["ndims"], E)
    F, M = dfr_numpy.wall_force(st, g.U0, wf, cfp, g.params, g.viscous)
    scale = np.abs(d["force"]).max()
    assert np.abs(F - d["force"]).max() <= 1e-12 * scale
    assert np.abs(M - d["moment"]).max() <= 1e-12 * max(np.abs(d["moment"]).max(), scale)


@pytest.mark.parametrize("name", gc.traj_names())
def test_oracle_first_step_matches_reference_trajectory(name):
    """One RK44 step of the restatement against the reference's first
    checkpoint (the supersonic case exercises inlet_sup, outlet_sup and
    wall_slip together)."""
    t = gc.load_traj(name)
    if t.meta["checkpoints"][0] != 1:
        pytest.skip("first checkpoint is not one step")
    from zefr_b200.solver import Plan, params_from_reference
    plan = Plan(t.mesh, params_from_reference(t.params, t.order), t.bounds)
    S, V, E = t.U0.shape
    st = dfr_numpy.Setup.from_arrays(t.meta["ndims"], S, plan.info.nfpts, E, plan.get)
    U1 = dfr_numpy.rk44_step(st, t.U0, t.params, t.viscous, t.meta["dt"])
    assert gc.rel_err(U1, t.states[0]) < 1e-12
