"""RK54 (fixed and adaptive dt) and RK44 with CFL time steps on the GPU
against the compiled reference's trajectories (tests/golden/time/*.npz):
dt(0) after every step, the per-element CFL steps and the final state.

Tolerances: plain FP64 form 1e-12 relative, except under the adaptive
controller (step sizes and states 1e-10): the embedded error estimate is a
combination of the five stage residuals that cancels to O(dt^5), so the
residual's summation-order rounding reaches the estimate -- and through
err^(-0.175) the next dt and every later state -- amplified.
Mixed form: states 1e-5 relative per variable and within 5% of the run's
change; CFL steps 1e-5; adaptive steps 1e-3 (the same cancellation acting on
the FP32 residual)."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200 import meshgen
from zefr_b200._lib import ZbError
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu

NAMES = gc.time_names()
TIME_KEYS = ("dt_type", "CFL", "CFL_type", "adapt_dt", "err_atol", "err_rtol", "pi_alpha", "pi_beta",
             "safety_factor", "max_factor", "min_factor", "max_dt")


def _solver(g, precision="fp64"):
    s = FRSolver(g.mesh, params_from_reference(g.params, g.order, precision=precision), g.bounds)
    s.set_time_scheme(g.deck.get("dt_scheme", "RK44"), **{k: v for k, v in g.deck.items() if k in TIME_KEYS})
    s.set_state(g.U0)
    return s


def _run(g, precision):
    s = _solver(g, precision)
    dts = []
    for _ in range(g.meta["nsteps"]):
        s.update()
        dts.append(s.time_state()["dt"])
    return s, np.array(dts)


@pytest.mark.parametrize("name", NAMES)
def test_time_integration_fp64_matches_reference(name):
    g = gc.load_time(name)
    s, dts = _run(g, "fp64")
    tol_dt = 1e-10 if g.deck.get("adapt_dt") else 1e-12
    assert np.max(np.abs(dts - g.dt0) / g.dt0) < tol_dt, (dts, g.dt0)
    assert gc.rel_err(s.get_state(), g.Un) < tol_dt
    if g.deck.get("dt_type", 0):
        dte = s.element_dt()
        assert np.max(np.abs(dte[1:] - g.dt_ele[1:]) / g.dt_ele[1:]) < 1e-12
    ts = s.time_state()
    assert ts["flow_time"] > 0
    if g.deck.get("adapt_dt"):
        assert 0 < ts["prev_err"] < 1
    s.close()


@pytest.mark.parametrize("name", ["rk54_quad_p3_vortex", "rk54_adapt_quad_p3_vortex", "cfl2_global_hex_p2_ns",
                                  "cfl1_global_quad_p2_ns"])
def test_time_integration_mixed(name):
    g = gc.load_time(name)
    s, dts = _run(g, "mixed")
    tol_dt = 1e-3 if g.deck.get("adapt_dt") else 1e-5
    assert np.max(np.abs(dts - g.dt0) / g.dt0) < tol_dt, (dts, g.dt0)
    U = s.get_state()
    assert gc.rel_err(U, g.Un) < 1e-5
    assert np.linalg.norm(U - g.Un) < 0.05 * np.linalg.norm(g.Un - g.U0)
    s.close()


def test_adaptive_counts_rejections():
    g = gc.load_time("rk54_adapt_quad_p3_vortex")
    s = _solver(g)
    s.update()
    assert s.time_state()["rejected"] >= 1
    s.close()


def test_time_scheme_errors():
    g = gc.load_time("rk54_quad_p3_vortex")
    s = FRSolver(g.mesh, params_from_reference(g.params, g.order), g.bounds)
    with pytest.raises(ZbError):
        s.set_time_scheme("RK44", adapt_dt=1)           # no embedded pair
    with pytest.raises(ZbError):
        s.set_time_scheme("RK54", dt_type=1)            # CFL steps are an RK44 option
    with pytest.raises(ValueError):
        s.set_time_scheme("RK33")
    s.set_time_scheme("RK54")
    s.set_state(g.U0)
    with pytest.raises(ZbError):
        s.step_RK_stage(0)                              # stage-wise stepping is RK44's
    s.close()
    tri = meshgen.box_tris(3, seed=1)
    gt = gc.load("tri_p2_euler_vortex")
    st = FRSolver(tri, params_from_reference(gt.params, 2), {"PERIODIC": "periodic"})
    with pytest.raises(ZbError):
        st.set_time_scheme("RK44", dt_type=1)
    st.close()


@pytest.mark.parametrize("name", ["rk54_adapt_quad_p3_vortex", "cfl2_global_hex_p2_ns"])
def test_from_deck_reproduces_reference_trajectory(name, tmp_path):
    """The same deck file the reference ran, read by FRSolver.from_deck."""
    from oracle import refcpu
    g = gc.load_time(name)
    meshgen.write_gmsh(g.mesh, str(tmp_path / "m.msh"))
    deck = refcpu.write_deck(str(tmp_path / "case.deck"), "m.msh", g.meta["ndims"], g.order, g.viscous, g.bounds,
                             g.deck)
    s = FRSolver.from_deck(deck)
    s.set_state(g.U0)
    dts = []
    for _ in range(g.meta["nsteps"]):
        s.update()
        dts.append(s.time_state()["dt"])
    tol = 1e-10 if g.deck.get("adapt_dt") else 1e-12
    assert np.max(np.abs(np.array(dts) - g.dt0) / g.dt0) < tol
    assert gc.rel_err(s.get_state(), g.Un) < tol
    s.close()


def test_checkpoint_resume_is_exact(tmp_path):
    """save_state / load_state: a resumed run continues bitwise like the
    uninterrupted one (plain FP64, RK54 at the fixed dt)."""
    from zefr_b200.output import load_state, save_state
    g = gc.load_time("rk54_quad_p3_vortex")
    a = _solver(g)
    a.update()
    save_state(str(tmp_path / "ck"), a)
    a.update()
    b = _solver(g)
    meta = load_state(str(tmp_path / "ck.npz"), b)
    assert meta["nspts"] == a.nspts and meta["time"]["flow_time"] > 0
    b.update()
    assert np.array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()
