"""Adjoint (vector-Jacobian product) of the residual against central finite
differences of the FP64 residual.

For a weight lam and a direction v, <Ubar, v> with Ubar = (dR/dU)^T lam must
equal <lam, (R(U + h v) - R(U - h v)) / 2h>; tolerance 1e-6 relative.  The
Rusanov flux has kinks (|Vn| and the max of the two wave speeds), which points
of the Taylor-Green state sit near, so the difference converges only about
linearly in h there: h = 1e-7 (relative to each variable's scale) keeps its
error near 1e-9, where h = 1e-6 leaves 1.6e-6.  The same check covers the
free-stream derivatives on far-field and characteristic faces."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu

TOL_FD = 1e-6
H = 1e-7

# every boundary kind, Euler and Navier-Stokes, quads, hexes and triangles
# (P1-P8), beta 0.5 and 0.3
CASES = ["quad_p1_euler", "quad_p3_euler_vortex", "quad_p5_euler", "quad_p2_ns_jitter", "hex_p1_ns",
         "hex_p2_euler_jitter", "hex_p3_ns_tgv", "cyl_p3_ns_char_adi", "cyl_p2_ns_iso_farfield_b03",
         "cyl_p3_euler_slip_char", "cyl_p2_euler_supin_sym", "tri_p1_ns_adi", "tri_p2_euler_vortex",
         "tri_p3_euler_char", "tri_p4_ns_jitter", "tri_p5_ns_jitter", "tri_p7_ns_adi", "tri_p8_euler_char"]


def solver_for(g, **kw):
    return FRSolver(g.mesh, params_from_reference(g.params, g.order, **kw), g.bounds)


def _directions(g, seed):
    rng = np.random.default_rng(seed)
    lam = rng.standard_normal(g.U0.shape)
    scale = np.abs(g.U0).max(axis=(0, 2))[None, :, None]
    v = rng.standard_normal(g.U0.shape) * scale
    return lam, v


@pytest.mark.parametrize("name", CASES)
def test_vjp_matches_central_differences(name):
    g = gc.load(name)
    s = solver_for(g)
    lam, v = _directions(g, 7)
    s.set_state(g.U0)
    Ubar = s.vjp(lam)
    lhs = float(np.sum(Ubar * v))
    Rp = s.residual(g.U0 + H * v)
    Rm = s.residual(g.U0 - H * v)
    rhs = float(np.sum(lam * (Rp - Rm)) / (2 * H))
    assert abs(lhs - rhs) <= TOL_FD * max(abs(rhs), 1e-300), (lhs, rhs)


@pytest.mark.parametrize("name", ["tri_p4_ns_jitter", "tri_p3_euler_char"])
def test_vjp_roe_matches_central_differences(name):
    """The Roe flux's reverse mode on triangles (the golden cases run the
    reference's Rusanov)."""
    g = gc.load(name)
    s = solver_for(g, fconv="roe")
    lam, v = _directions(g, 13)
    s.set_state(g.U0)
    lhs = float(np.sum(s.vjp(lam) * v))
    rhs = float(np.sum(lam * (s.residual(g.U0 + H * v) - s.residual(g.U0 - H * v))) / (2 * H))
    assert abs(lhs - rhs) <= TOL_FD * max(abs(rhs), 1e-300), (lhs, rhs)


def test_vjp_geometry_rejected_on_triangles():
    from zefr_b200._lib import ZbError
    g = gc.load("tri_p2_euler_vortex")
    s = solver_for(g)
    s.set_state(g.U0)
    with pytest.raises(ZbError) as ei:
        s.vjp_geometry(np.ones(g.U0.shape))
    assert ei.value.status == -4


@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "cyl_p2_ns_iso_farfield_b03", "cyl_p3_euler_slip_char",
                                  "cyl_p2_euler_supin_sym", "tri_p3_euler_char", "tri_p8_euler_char"])
def test_vjp_freestream_matches_central_differences(name):
    g = gc.load(name)
    s = solver_for(g)
    lam, _ = _directions(g, 11)
    s.set_state(g.U0)
    _, pbar = s.vjp(lam, params=True)
    p = g.params
    base = dict(rho_fs=p["rho_fs"], V_fs=[p["V_fs0"], p["V_fs1"], p["V_fs2"]], P_fs=p["P_fs"])
    for k in range(5):
        if 1 <= k <= 3 and k > g.meta["ndims"]:
            continue
        res = []
        for sgn in (1.0, -1.0):
            kw = {"rho_fs": base["rho_fs"], "V_fs": list(base["V_fs"]), "P_fs": base["P_fs"]}
            if k == 0:
                step = H * max(1.0, abs(kw["rho_fs"]))
                kw["rho_fs"] += sgn * step
            elif k <= 3:
                step = H * max(1.0, abs(kw["V_fs"][k - 1]))
                kw["V_fs"][k - 1] += sgn * step
            else:
                step = H * max(1.0, abs(kw["P_fs"]))
                kw["P_fs"] += sgn * step
            kw["V_fs"] = tuple(kw["V_fs"])
            res.append(solver_for(g, **kw).residual(g.U0))
        fd = float(np.sum(lam * (res[0] - res[1])) / (2 * step))
        scale = max(abs(fd), 1e-8 * float(np.abs(lam).sum()))
        assert abs(pbar[k] - fd) <= TOL_FD * scale + 1e-9, (k, pbar[k], fd)


def test_vjp_is_deterministic_and_linear():
    g = gc.load("cyl_p3_ns_char_adi")
    s = solver_for(g)
    lam, _ = _directions(g, 3)
    s.set_state(g.U0)
    a = s.vjp(lam)
    b = s.vjp(lam)
    c = s.vjp(2.0 * lam)
    assert np.array_equal(a, b)
    assert np.array_equal(c, 2.0 * a)


def test_vjp_device_tensors():
    torch = pytest.importorskip("torch")
    g = gc.load("hex_p3_ns_tgv")
    s = solver_for(g)
    lam, _ = _directions(g, 5)
    s.set_state(g.U0)
    host = s.vjp(lam)
    dev = s.vjp(torch.from_numpy(lam).cuda())
    assert dev.is_cuda
    assert np.array_equal(dev.cpu().numpy(), host)


def test_vjp_rejects_mixed_form():
    g = gc.load("quad_p3_euler_vortex")
    s = solver_for(g, precision="mixed")
    s.set_state(g.U0)
    with pytest.raises(RuntimeError, match="FP64"):
        s.vjp(np.zeros(g.U0.shape))
