"""Geometry adjoint of the residual and the cylinder drag gradient against
central finite differences (FP64).

Residual level: for a fixed state U and weight lam, d(lam . R)/d(node
coordinates) from zb_vjp_geometry chained through the torch restatement of
the metrics must equal the central difference of lam . R under a random node
displacement (interior nodes only on periodic meshes, so periodic faces stay
paired).  Trajectory level: the mean drag over RK44 steps on a small curved
cylinder mesh, differentiated with respect to wall Fourier coefficients and
the free-stream angle, against central differences of the forward run."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200.meshgen import Mesh
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from zefr_b200 import geometry  # noqa: E402
from zefr_b200.shape import CylinderDrag  # noqa: E402

TOL = 1e-6


def _displaced(mesh, delta):
    return Mesh(mesh.ndims, np.asarray(mesh.nodes) + delta, mesh.gmsh_type, mesh.elements, mesh.bnd_faces)


def _interior_nodes(mesh):
    on_bnd = np.zeros(len(mesh.nodes), dtype=bool)
    for f in mesh.bnd_faces:
        on_bnd[list(f[1])] = True
    return ~on_bnd


@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "cyl_p3_euler_slip_char", "quad_p2_ns_jitter",
                                  "hex_p2_euler_jitter", "cyl_p2_ns_iso_farfield_b03", "hex_p1_ns", "hex_p3_ns_tgv"])
def test_geometry_adjoint_matches_central_differences(name):
    g = gc.load(name)
    D = g.meta["ndims"]
    p = params_from_reference(g.params, g.order)
    rng = np.random.default_rng(3)
    lam = rng.standard_normal(g.U0.shape)
    delta = np.zeros((len(g.mesh.nodes), 3))
    move = np.ones(len(g.mesh.nodes), dtype=bool) if name.startswith("cyl") else _interior_nodes(g.mesh)
    delta[move, :D] = rng.standard_normal((int(move.sum()), D))
    U = g.U0.copy()
    if name.startswith("cyl"):
        # The fixture's stream is along x with exactly zero y-momentum, so at
        # far-field points whose normal is vertical the normal velocity is
        # zero to rounding: |Vn| and the characteristic inflow/outflow switch
        # have kinks there and a difference quotient has no derivative to
        # match.  Turn the stream by 0.5 rad to move off them.
        c, sn = np.cos(0.5), np.sin(0.5)
        mx, my = U[:, 1].copy(), U[:, 2].copy()
        U[:, 1], U[:, 2] = c * mx - sn * my, sn * mx + c * my
    elif D == 3:
        # The hexahedral fixtures hold Taylor-Green-like states with w = 0
        # everywhere, so the normal velocity at every z-face point is exactly
        # zero: the Rusanov flux's |Vn| has its kink there and the residual
        # has no derivative with respect to the face normal (central
        # differences then differ from the adjoint by a constant, whatever
        # the step).  Turn the velocity by 0.5 rad about x, then about z.
        c, sn = np.cos(0.5), np.sin(0.5)
        my, mz = U[:, 2].copy(), U[:, 3].copy()
        U[:, 2], U[:, 3] = c * my - sn * mz, sn * my + c * mz
        mx, my = U[:, 1].copy(), U[:, 2].copy()
        U[:, 1], U[:, 2] = c * mx - sn * my, sn * mx + c * my
    s = FRSolver(g.mesh, p, g.bounds)
    s.set_state(U)
    _, _, bars = s.vjp_geometry(lam)
    gm = geometry.GeometryMap(s, g.mesh)
    X = gm.nodes0.clone().requires_grad_(True)
    m = gm.metrics(X)
    keys = list(m)
    gX = torch.autograd.grad([m[k] for k in keys], X,
                             grad_outputs=[torch.from_numpy(bars[k]).cuda() for k in keys])[0].cpu().numpy()
    lhs = float((gX * delta[:, :D]).sum())
    h = 1e-7
    vals = []
    for sgn in (1.0, -1.0):
        sp = FRSolver(_displaced(g.mesh, sgn * h * delta), p, g.bounds)
        vals.append(float((lam * sp.residual(U, 0)).sum()))
        sp.close()
    rhs = (vals[0] - vals[1]) / (2 * h)
    assert abs(lhs - rhs) <= TOL * abs(rhs), (lhs, rhs)


def test_cylinder_drag_gradient_matches_central_differences():
    prob = CylinderDrag(nr=5, nt=12, order=2, r1=6.0, ncoef=4, dt=2e-4, checkpoint_every=2)
    coef = np.array([0.01, -0.005, 0.003, 0.002])
    alpha, nsteps = 0.1, 6
    out = prob.gradient(coef, alpha, nsteps)
    J0 = prob.drag(coef, alpha, nsteps)
    assert abs(out["J"] - J0) <= 1e-12 * abs(J0)
    h = 1e-6
    for k in range(len(coef)):
        cp, cm = coef.copy(), coef.copy()
        cp[k] += h
        cm[k] -= h
        fd = (prob.drag(cp, alpha, nsteps) - prob.drag(cm, alpha, nsteps)) / (2 * h)
        assert abs(out["dJ_dcoef"][k] - fd) <= TOL * max(abs(fd), 1e-3 * abs(J0)), (k, out["dJ_dcoef"][k], fd)
    fd = (prob.drag(coef, alpha + h, nsteps) - prob.drag(coef, alpha - h, nsteps)) / (2 * h)
    assert abs(out["dJ_dalpha"] - fd) <= TOL * max(abs(fd), 1e-3 * abs(J0)), (out["dJ_dalpha"], fd)
