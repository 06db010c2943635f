"""VTU output (plot-point interpolation, sub-cells, fields) and the raw
state checkpoint, on host-side plans (no GPU)."""
import numpy as np
import pytest

from zefr_b200 import meshgen
from zefr_b200.output import read_vtu_array, write_vtu
from zefr_b200.solver import Plan, make_params


def _linear_state(X, D):
    """rho, momentum and energy linear in x: plot-point interpolation of a
    degree >= 1 polynomial basis reproduces it exactly."""
    S, _, E = X.shape
    U = np.zeros((S, D + 2, E))
    U[:, 0] = 1.0 + 0.1 * X[:, 0]
    U[:, 1] = 0.3 + 0.05 * X[:, 1 % D]
    U[:, D + 1] = 2.5 + 0.01 * X[:, 0]
    return U


@pytest.mark.parametrize("case", ["quad_p3", "hex_p2", "cyl_p3_quad9"])
def test_vtu_plot_points_and_fields(case, tmp_path):
    if case == "quad_p3":
        mesh, order, bnd = meshgen.box_quads(3, 2), 3, {"PERIODIC": "periodic"}
    elif case == "hex_p2":
        mesh, order, bnd = meshgen.box_hexes(2, 2, 1), 2, {"PERIODIC": "periodic"}
    else:
        mesh, order, bnd = meshgen.cylinder_omesh(2, 8, r1=3.0), 3, {"WALL": "wall_slip", "FARFIELD": "char"}
    plan = Plan(mesh, make_params(order, False), bnd)
    D, S, E = mesh.ndims, plan.info.nspts, plan.info.n_eles
    X = plan.get("coord_spts").reshape(S, D, E)
    U = _linear_state(X, D)
    path = str(tmp_path / "sol.vtu")
    write_vtu(path, plan, U)
    P = order + 3
    pts = read_vtu_array(path, "Points")
    assert pts.shape == (E * P ** D, 3)
    conn = read_vtu_array(path, "connectivity")
    assert len(conn) == E * (P - 1) ** D * 2 ** D and conn.max() == E * P ** D - 1
    rho = read_vtu_array(path, "Density")
    assert np.allclose(rho, 1.0 + 0.1 * pts[:, 0], atol=1e-12)
    vel = read_vtu_array(path, "Velocity")
    assert np.allclose(vel[:, 0] * rho, 0.3 + 0.05 * pts[:, 1 % D], atol=1e-12)
    if case != "cyl_p3_quad9":
        # element corners of linear elements land on mesh nodes
        corners = pts.reshape(E, P ** D, 3)[:, 0, :D]
        d = np.abs(corners[:, None, :] - np.asarray(mesh.nodes)[None, :, :D]).max(-1).min(1)
        assert d.max() < 1e-12


def test_vtu_triangles_are_points(tmp_path):
    mesh = meshgen.box_tris(3, seed=1)
    plan = Plan(mesh, make_params(2, False), {"PERIODIC": "periodic"})
    S, E = plan.info.nspts, plan.info.n_eles
    X = plan.get("coord_spts").reshape(S, 2, E)
    path = str(tmp_path / "tri.vtu")
    write_vtu(path, plan, _linear_state(X, 2))
    assert read_vtu_array(path, "Points").shape == (S * E, 3)
    assert set(read_vtu_array(path, "types").tolist()) == {1}
