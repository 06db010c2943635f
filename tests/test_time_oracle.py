"""The numpy restatement of the reference's time integration (RK54 with and
without the adaptive controller, RK44 with CFL time steps) against the
compiled reference's own trajectories (tests/golden/time/*.npz).  CPU only:
the set-up arrays come from the host-side plan, which test_setup.py pins to
the reference."""
import numpy as np
import pytest

import golden_cases as gc
from oracle import dfr_numpy
from zefr_b200.solver import Plan, params_from_reference

NAMES = gc.time_names()
TOL = 1e-12


def test_time_fixtures_present():
    assert len(NAMES) >= 6


def _setup(g):
    plan = Plan(g.mesh, params_from_reference(g.params, g.order), g.bounds)
    S, V, E = g.U0.shape
    st = dfr_numpy.Setup.from_arrays(g.mesh.ndims, S, plan.info.nfpts, E, plan.get)
    return plan, st


def _cfl_geometry(plan, st, g):
    S, V, E = g.U0.shape
    D = g.mesh.ndims
    Fp = plan.info.nfpts
    N = g.order + 1
    w1 = np.polynomial.legendre.leggauss(N)[1]
    wf = w1 if D == 2 else np.outer(w1, w1).reshape(-1)
    vol = (plan.get("weights_spts")[:, None] * st.jaco_det).sum(0)
    href = dfr_numpy.h_ref(plan.get("coord_fpts").reshape(Fp, D, E), plan.get("loc_fpts").reshape(Fp, D),
                           Fp // (2 * D))
    return vol, wf, href


@pytest.mark.parametrize("name", NAMES)
def test_oracle_time_integration_matches_reference(name):
    g = gc.load_time(name)
    deck = g.deck
    plan, st = _setup(g)
    U = g.U0.copy()
    dts = []
    if deck.get("dt_scheme") == "RK54":
        if deck.get("adapt_dt"):
            ctl = dfr_numpy.AdaptiveRK54(deck["dt"], atol=deck.get("err_atol", 1e-5), rtol=deck.get("err_rtol", 1e-5))
            for _ in range(g.meta["nsteps"]):
                U = ctl.step(st, U, g.params, g.viscous)
                dts.append(ctl.dt)
        else:
            for _ in range(g.meta["nsteps"]):
                U, _ = dfr_numpy.lsrk_step(st, U, g.params, g.viscous, deck["dt"])
                dts.append(deck["dt"])
    else:
        vol, wf, href = _cfl_geometry(plan, st, g)
        for _ in range(g.meta["nsteps"]):
            dte = dfr_numpy.element_dt(st, U, g.params, g.viscous, g.order, deck["CFL"], deck["CFL_type"], vol, wf,
                                       href)
            dt = dte.min() if deck["dt_type"] == 1 else dte
            U = dfr_numpy.rk44_step_dt(st, U, g.params, g.viscous, dt)
            dts.append(float(dte.min() if deck["dt_type"] == 1 else dte[0]))
        # the reference keeps the per-element estimates of the last step,
        # with element 0's replaced by the global minimum under dt_type 1
        ref = g.dt_ele.copy()
        assert np.max(np.abs(ref[1:] - dte[1:]) / np.abs(ref[1:])) < TOL
    assert np.max(np.abs(np.array(dts) - g.dt0) / np.abs(g.dt0)) < TOL, (dts, g.dt0)
    assert gc.rel_err(U, g.Un) < TOL


def test_adaptive_fixture_rejects_a_step():
    """The large initial dt of the adaptive vortex case forces rejections."""
    g = gc.load_time("rk54_adapt_quad_p3_vortex")
    _, st = _setup(g)
    ctl = dfr_numpy.AdaptiveRK54(g.deck["dt"])
    ctl.step(st, g.U0, g.params, g.viscous)
    assert ctl.rejected >= 1


def test_oracle_detects_planted_time_error():
    """A wrong embedded weight in the oracle must change the dt sequence."""
    g = gc.load_time("rk54_adapt_quad_p3_vortex")
    _, st = _setup(g)
    saved = list(dfr_numpy.LSRK_BHAT)
    try:
        dfr_numpy.LSRK_BHAT[4] *= 1.0001
        ctl = dfr_numpy.AdaptiveRK54(g.deck["dt"])
        U = g.U0
        for _ in range(g.meta["nsteps"]):
            U = ctl.step(st, U, g.params, g.viscous)
        assert abs(ctl.dt - g.dt0[-1]) > 1e-9 * g.dt0[-1]
    finally:
        dfr_numpy.LSRK_BHAT[:] = saved
