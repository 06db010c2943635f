"""Torch restatements used by the shape adjoint, on the CPU: the set-up
metrics as functions of the node coordinates (the checker of the library's
geometry kernels) must reproduce the plan's, and the wall force must equal
the oracle's compute_moments restatement."""
import numpy as np
import pytest

import golden_cases as gc
from oracle import dfr_numpy
from zefr_b200.solver import Plan, make_params

torch = pytest.importorskip("torch")

from zefr_b200 import geometry  # noqa: E402
from geometry_restatement import GeometryRestatement  # noqa: E402


class _PlanView:
    """The parts of FRSolver the torch restatements read, from a host Plan."""

    def __init__(self, g):
        self.plan = Plan(g.mesh, make_params(g.order, g.viscous), g.bounds)
        self.info = self.plan.info
        self.ndims = self.info.ndims
        self.nspts, self.nvars, self.neles = self.info.nspts, self.info.nvars, int(self.info.n_eles)


@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "quad_p2_ns_jitter", "hex_p2_euler_jitter",
                                  "tri_p3_euler_char", "tri_p4_ns_jitter"])
def test_geometry_map_reproduces_plan_metrics(name):
    g = gc.load(name)
    v = _PlanView(g)
    gm = GeometryRestatement(v, g.mesh, device="cpu")
    m = gm.metrics(gm.nodes0)
    for key, arr in (("inv_jaco", "inv_jaco_spts"), ("jaco_det", "jaco_det_spts"), ("norm", "fpt_norm"),
                     ("dA", "fpt_dA")):
        a = m[key].numpy().reshape(-1)
        b = v.plan.get(arr)
        assert np.abs(a - b).max() <= 1e-13 * max(1.0, np.abs(b).max()), key


@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "cyl_p2_ns_iso_farfield_b03", "cyl_p3_euler_slip_char"])
def test_torch_wall_force_matches_oracle(name):
    g = gc.load(name)
    v = _PlanView(g)
    gm = GeometryRestatement(v, g.mesh, device="cpu")
    wf = geometry.WallForce(v, g.params, device="cpu")
    F = wf.force(torch.from_numpy(g.U0), gm.metrics(gm.nodes0)).numpy()
    st = g.setup()
    N = g.order + 1
    w1 = np.polynomial.legendre.leggauss(N)[1]
    Fp = st.oppE.shape[0]
    S, V, E = g.U0.shape
    cfp = v.plan.get("coord_fpts").reshape(Fp, 2, E)
    Fo, _ = dfr_numpy.wall_force(st, g.U0, np.array([w1[f % N] for f in range(Fp)]), cfp, g.params, g.viscous)
    assert np.abs(F - Fo[:2]).max() <= 1e-12 * np.abs(Fo).max()


@pytest.mark.parametrize("name", ["cyl_p3_ns_char_adi", "hex_p2_euler_jitter", "tri_p3_euler_char"])
def test_plan_nodes_and_shape_tables_give_the_coordinates(name):
    """The element nodes and solution-point shape functions the plan exports
    (inputs of the device geometry kernels) reproduce its solution-point
    coordinates bit for bit when summed in node order, as the set-up does."""
    g = gc.load(name)
    v = _PlanView(g)
    D, S, E = v.ndims, v.nspts, v.neles
    nodes = v.plan.get("nodes").reshape(-1, D, E)
    nn = nodes.shape[0]
    sh = v.plan.get("shape_spts").reshape(S, nn)
    X = np.zeros((S, D, E))
    for n in range(nn):
        X += sh[:, n][:, None, None] * nodes[n][None, :, :]
    assert np.array_equal(X.reshape(-1), v.plan.get("coord_spts"))
    # the element nodes are the mesh nodes each element names, in gmsh order
    mesh_nodes = np.asarray(g.mesh.nodes)[:, :D]
    e2n = np.asarray(g.mesh.elements)
    assert np.array_equal(nodes, mesh_nodes[e2n].transpose(1, 2, 0))
