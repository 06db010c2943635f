"""Geometry kernels (zb_geometry_eval, zb_geometry_eval_vjp, zb_set_nodes):
the metrics of the element nodes equal the host set-up's bit for bit, their
adjoint equals torch autograd through the restatement of the set-up, and a
moved context gives the residual, wall force and CFL step of a solver built
on the moved mesh."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200._lib import ZbError
from zefr_b200.meshgen import Mesh
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from geometry_restatement import GeometryRestatement  # noqa: E402
from zefr_b200 import geometry  # noqa: E402

CASES = ["cyl_p3_ns_char_adi", "quad_p2_ns_jitter", "hex_p2_euler_jitter", "hex_p3_ns_tgv", "tri_p3_euler_char",
         "tri_p4_ns_jitter", "quad_p5_euler"]
PLAN_NAMES = {"inv_jaco": "inv_jaco_spts", "jaco_det": "jaco_det_spts", "norm": "fpt_norm", "dA": "fpt_dA"}


def solver_for(g, mesh=None, **kw):
    return FRSolver(mesh if mesh is not None else g.mesh, params_from_reference(g.params, g.order, **kw), g.bounds)


def _displaced(mesh, delta):
    return Mesh(mesh.ndims, np.asarray(mesh.nodes) + delta, mesh.gmsh_type, mesh.elements, mesh.bnd_faces)


def _smooth_motion(mesh, amp):
    """A smooth displacement field, small against the element size."""
    X = np.asarray(mesh.nodes)
    D = mesh.ndims
    lo, hi = X[:, :D].min(axis=0), X[:, :D].max(axis=0)
    r = (X[:, :D] - lo) / np.maximum(hi - lo, 1e-30)
    delta = np.zeros_like(X)
    for d in range(D):
        delta[:, d] = amp * (hi[d] - lo[d]) * np.sin(np.pi * r[:, d]) * np.sin(2.0 * np.pi * r[:, (d + 1) % D])
    return delta


@pytest.mark.parametrize("name", CASES)
def test_geometry_eval_equals_setup_bitwise(name):
    g = gc.load(name)
    s = solver_for(g)
    nodes = torch.from_numpy(s.plan.get("nodes").reshape(s.nodes_shape)).cuda()
    m = s.geometry_eval(nodes)
    for k, pn in PLAN_NAMES.items():
        assert np.array_equal(m[k].cpu().numpy().reshape(-1), s.plan.get(pn)), k
    # the element nodes gathered from the mesh are the plan's
    gm = geometry.GeometryMap(s, g.mesh)
    assert torch.equal(gm.element_nodes(gm.nodes0), nodes)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_geometry_eval_vjp_matches_restatement_autograd(name):
    """Node adjoint against torch autograd through the restated set-up, for
    random adjoints of all four arrays (different summation order: 1e-12)."""
    g = gc.load(name)
    s = solver_for(g)
    rng = np.random.default_rng(7)
    shapes = s._geometry_shapes()
    bars = {k: torch.from_numpy(rng.standard_normal(sh)).cuda() for k, sh in shapes.items()}
    nodes = torch.from_numpy(s.plan.get("nodes").reshape(s.nodes_shape)).cuda()
    got = s.geometry_eval_vjp(nodes, bars).cpu().numpy()
    rs = GeometryRestatement(s, g.mesh)
    X = rs.nodes0.clone().requires_grad_(True)
    m = rs.metrics(X)
    gX = torch.autograd.grad([m[k] for k in shapes], X, grad_outputs=[bars[k] for k in shapes])[0]
    # the kernel's node adjoint per element node, summed to mesh nodes
    e2n = torch.as_tensor(np.asarray(g.mesh.elements, dtype=np.int64))
    D = s.ndims
    ref = gX.cpu().numpy()
    mine = np.zeros_like(ref)
    np.add.at(mine, e2n.numpy().T.reshape(-1), got.transpose(0, 2, 1).reshape(-1, D))
    scale = np.abs(ref).max()
    assert np.abs(mine - ref).max() <= 1e-12 * scale
    # one array at a time: a missing adjoint counts as zero
    for k in shapes:
        one = s.geometry_eval_vjp(nodes, {k: bars[k]}).cpu().numpy()
        m = rs.metrics(X)
        gk = torch.autograd.grad(m[k], X, grad_outputs=bars[k])[0].cpu().numpy()
        mk = np.zeros_like(gk)
        np.add.at(mk, e2n.numpy().T.reshape(-1), one.transpose(0, 2, 1).reshape(-1, D))
        assert np.abs(mk - gk).max() <= 1e-12 * max(np.abs(gk).max(), 1e-300), k
    s.close()


def test_geometry_eval_vjp_is_deterministic_and_linear():
    g = gc.load("hex_p2_euler_jitter")
    s = solver_for(g)
    rng = np.random.default_rng(2)
    bars = {k: torch.from_numpy(rng.standard_normal(sh)).cuda() for k, sh in s._geometry_shapes().items()}
    nodes = torch.from_numpy(s.plan.get("nodes").reshape(s.nodes_shape)).cuda()
    a = s.geometry_eval_vjp(nodes, bars)
    b = s.geometry_eval_vjp(nodes, bars)
    assert torch.equal(a, b)
    two = s.geometry_eval_vjp(nodes, {k: 2.0 * v for k, v in bars.items()})
    assert torch.equal(two, 2.0 * a)
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "hex_p2_euler_jitter", "tri_p4_ns_jitter"])
def test_set_nodes_equals_solver_on_moved_mesh(name, precision):
    g = gc.load(name)
    moved = _displaced(g.mesh, _smooth_motion(g.mesh, 0.01))
    s = solver_for(g, precision=precision)
    fresh = solver_for(g, moved, precision=precision)
    before = s.residual(g.U0, 0)
    s.set_nodes(fresh.plan.get("nodes").reshape(s.nodes_shape))
    after = s.residual(g.U0, 0)
    want = fresh.residual(g.U0, 0)
    assert np.array_equal(after, want)
    assert not np.array_equal(before, want)
    # from device tensors: back to the set-up mesh (the plan handle keeps
    # it), then the move again
    s.set_nodes(torch.from_numpy(s.plan.get("nodes").reshape(s.nodes_shape)).cuda())
    assert np.array_equal(s.residual(g.U0, 0), before)
    s.set_nodes(torch.from_numpy(fresh.plan.get("nodes").reshape(s.nodes_shape)).cuda())
    assert np.array_equal(s.residual(g.U0, 0), want)
    if name.startswith("cyl"):
        s.set_state(g.U0)
        fresh.set_state(g.U0)
        a, b = s.wall_force(), fresh.wall_force()
        for k in a:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    s.close()
    fresh.close()


def test_set_nodes_refreshes_cfl_step():
    g = gc.load("quad_p2_ns_jitter")
    moved = _displaced(g.mesh, _smooth_motion(g.mesh, 0.02))
    s = solver_for(g)
    fresh = solver_for(g, moved)
    for sv in (s, fresh):
        sv.set_time_scheme("RK44", dt_type=2, CFL_type=2, CFL=0.5)
    s.set_nodes(fresh.plan.get("nodes").reshape(s.nodes_shape))
    for sv in (s, fresh):
        sv.set_state(g.U0)
        sv.step(1)
    assert np.array_equal(s.element_dt(), fresh.element_dt())
    assert np.array_equal(s.get_state(), fresh.get_state())
    s.close()
    fresh.close()


def test_set_nodes_rejects_inverted_mesh_and_keeps_geometry():
    g = gc.load("quad_p2_ns_jitter")
    s = solver_for(g)
    before = s.residual(g.U0, 0)
    nodes = s.plan.get("nodes").reshape(s.nodes_shape).copy()
    nodes[:, 0, :] *= -1.0  # mirror x: every element turns inside out
    with pytest.raises(ZbError):
        s.set_nodes(nodes)
    assert np.array_equal(s.residual(g.U0, 0), before)
    s.close()
