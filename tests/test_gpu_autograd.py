"""torch.autograd over the residual and the checkpointed RK44 trajectory
adjoint, against central differences (FP64)."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from zefr_b200 import autograd as zag  # noqa: E402

TOL_FD = 1e-6


def solver_for(g, **kw):
    return FRSolver(g.mesh, params_from_reference(g.params, g.order, **kw), g.bounds)


def test_residual_backward_is_the_library_adjoint():
    g = gc.load("cyl_p3_ns_char_adi")
    s = solver_for(g)
    rng = np.random.default_rng(1)
    lam = torch.from_numpy(rng.standard_normal(g.U0.shape)).cuda()
    U = torch.from_numpy(g.U0).cuda().requires_grad_(True)
    R = zag.residual(U, s)
    assert np.allclose(R.detach().cpu().numpy(), s.residual(g.U0), rtol=0, atol=0)
    (R * lam).sum().backward()
    s.set_state(g.U0)
    ref = s.vjp(lam.cpu().numpy())
    assert np.array_equal(U.grad.cpu().numpy(), ref)


@pytest.mark.parametrize("name", ["quad_p3_euler_vortex", "cyl_p3_ns_char_adi", "tri_p4_ns_jitter"])
def test_rk_step_vjp_equals_composed_stage_adjoints(name):
    """zb_rk_step_vjp against the RK44 transpose written out here from the
    residual adjoint (zb_vjp) and the stage tables of src/solver.cpp:722-735:
    U_{s+1} = U_0 - a_s dt/|J| R(U_s), U_new = U_0 - dt/|J| sum_s b_s R(U_s).
    Same kernels in a different order of sums: 1e-12 relative."""
    g = gc.load(name)
    s = solver_for(g)
    dt = 1e-3 if "vortex" in name else 2e-4
    s.set_dt(dt)
    S, V, E = s.state_shape
    inv_det = torch.from_numpy(1.0 / s.plan.get("jaco_det_spts").reshape(S, 1, E)).cuda()
    alpha, beta = (0.5, 0.5, 1.0), (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
    U0 = torch.from_numpy(g.U0).cuda()
    Us = [U0]
    for a in alpha:
        Us.append(U0 - a * dt * inv_det * zag.residual(Us[-1], s))
    rng = np.random.default_rng(11)
    ub = torch.from_numpy(rng.standard_normal(g.U0.shape)).cuda()
    ub0, ub_next, pref = ub.clone(), None, np.zeros(5)
    for st in range(3, -1, -1):
        lam = -beta[st] * dt * inv_det * ub
        if ub_next is not None:
            lam = lam - alpha[st] * dt * inv_det * ub_next
        s.set_state(Us[st])
        ubs, p = s.vjp(lam.contiguous(), params=True)
        pref += p
        ub0 = ub0 + ubs
        ub_next = ubs
    pbar = np.zeros(5)
    got = s.rk_step_vjp(U0, ub, pbar)
    ref = ub0.cpu().numpy()
    err = np.abs(got.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err <= 1e-12, err
    assert np.allclose(pbar, pref, rtol=1e-12, atol=1e-12 * np.abs(pref).max())


def _fd_objective(traj, U0, v, h, nsteps, obj):
    vals = []
    for sgn in (1.0, -1.0):
        U = torch.from_numpy(U0 + sgn * h * v).cuda()
        J = 0.0
        with torch.no_grad():
            for _ in range(nsteps):
                U = traj._step(U)
                J += float(obj(U))
        vals.append(J / nsteps)
    return (vals[0] - vals[1]) / (2 * h)


@pytest.mark.parametrize("name,every", [("quad_p3_euler_vortex", 2), ("cyl_p3_ns_char_adi", 3)])
def test_trajectory_adjoint_matches_central_differences(name, every):
    g = gc.load(name)
    s = solver_for(g)
    dt = 1e-3 if "vortex" in name else 2e-4
    nsteps = 6
    traj = zag.TrajectoryAdjoint(s, dt, checkpoint_every=every)
    obj = zag.kinetic_energy(s)
    out = traj.run(g.U0, nsteps, obj)
    rng = np.random.default_rng(4)
    scale = np.abs(g.U0).max(axis=(0, 2))[None, :, None]
    v = rng.standard_normal(g.U0.shape) * scale
    lhs = float((out["dJ_dU0"].cpu().numpy() * v).sum())
    rhs = _fd_objective(traj, g.U0, v, 1e-7, nsteps, obj)
    assert abs(lhs - rhs) <= TOL_FD * abs(rhs), (lhs, rhs)


def test_trajectory_freestream_gradient_matches_central_differences():
    g = gc.load("cyl_p3_euler_slip_char")
    s = solver_for(g)
    p = g.params
    rho, V, P = p["rho_fs"], [p["V_fs0"], p["V_fs1"], p["V_fs2"]], p["P_fs"]
    traj = zag.TrajectoryAdjoint(s, 2e-4, checkpoint_every=2)
    obj = zag.kinetic_energy(s)
    nsteps = 4
    out = traj.run(g.U0, nsteps, obj)
    for k, h in ((0, 1e-5), (1, 1e-5), (2, 1e-5), (4, 1e-5)):
        vals = []
        for sgn in (1.0, -1.0):
            rr, VV, PP = rho, list(V), P
            if k == 0:
                rr += sgn * h
            elif k <= 3:
                VV[k - 1] += sgn * h
            else:
                PP += sgn * h
            s.set_freestream(rr, VV, PP)
            U = torch.from_numpy(g.U0).cuda()
            J = 0.0
            with torch.no_grad():
                for _ in range(nsteps):
                    U = traj._step(U)
                    J += float(obj(U))
            vals.append(J / nsteps)
        s.set_freestream(rho, V, P)
        fd = (vals[0] - vals[1]) / (2 * h)
        got = out["dJ_dfreestream"][k]
        assert abs(got - fd) <= TOL_FD * abs(fd) + 1e-9, (k, got, fd)
