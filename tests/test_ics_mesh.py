"""Host-side workload definitions, on the CPU: the initial conditions the
benchmarks and tests start from, and the cylinder O-mesh whose node
positions the drag gradient differentiates (it must be affine in the wall
coefficients, since the gradient sums node adjoints against one displacement
field per coefficient), and the seeded parameters of the batched workload."""
import math

import numpy as np

from zefr_b200 import ics, meshgen
from zefr_b200.shape import CylinderDrag


def _grid(D, n=6, lo=0.0, hi=2 * math.pi, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(n, D, 5))  # (S, D, E)


def _primitive(U, gamma=1.4):
    D = U.shape[1] - 2
    rho = U[:, 0]
    vel = [U[:, d + 1] / rho for d in range(D)]
    p = (gamma - 1.0) * (U[:, D + 1] - 0.5 * rho * sum(v * v for v in vel))
    return rho, vel, p


def test_taylor_green_fields():
    X = _grid(3)
    mach, g = 0.1, 1.4
    U = ics.taylor_green(X, mach=mach, gamma=g)
    rho, (u, v, w), p = _primitive(U, g)
    U0 = mach * math.sqrt(g)
    x, y, z = X[:, 0], X[:, 1], X[:, 2]
    assert np.allclose(u, U0 * np.sin(x) * np.cos(y) * np.cos(z), rtol=0, atol=1e-14)
    assert np.allclose(v, -U0 * np.cos(x) * np.sin(y) * np.cos(z), rtol=0, atol=1e-14)
    assert np.array_equal(w, np.zeros_like(w))
    pw = 1.0 + U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    assert np.allclose(p, pw, rtol=1e-13, atol=0)
    assert np.allclose(rho, pw, rtol=1e-13, atol=0)  # rho = p rho0 / p0 with rho0 = p0 = 1


def test_isentropic_vortex_is_isentropic_with_its_core_temperature():
    X = _grid(2, lo=-5.0, hi=5.0)
    g, beta = 1.4, 5.0
    U = ics.isentropic_vortex(X, beta=beta, gamma=g)
    rho, _, p = _primitive(U, g)
    assert np.allclose(p / rho ** g, 1.0, rtol=1e-12, atol=0)
    core = ics.isentropic_vortex(np.zeros((1, 2, 1)), beta=beta, gamma=g)
    rc, vc, pc = _primitive(core, g)
    T = pc / rc
    assert abs(T.item() - (1.0 - (g - 1.0) * beta ** 2 / (8.0 * g * math.pi ** 2) * math.e)) < 1e-14
    assert abs(vc[0].item() - 1.0) < 1e-14 and abs(vc[1].item()) < 1e-14


def test_double_shear_layer_is_seeded_and_bounded():
    X = _grid(2, lo=0.0, hi=1.0)
    a = ics.double_shear_layer(X, noise=1e-3, seed=7)
    b = ics.double_shear_layer(X, noise=1e-3, seed=7)
    c = ics.double_shear_layer(X, noise=1e-3, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    clean = ics.double_shear_layer(X, noise=0.0)
    U0 = 0.2 * math.sqrt(1.4)
    du = np.abs(a[:, 1] - clean[:, 1])  # rho = 1
    assert du.max() <= 1e-3 * U0 * (1 + 1e-12)
    rho, _, p = _primitive(clean)
    assert np.allclose(rho, 1.0) and np.allclose(p, 1.0, rtol=1e-13)


def test_cylinder_mesh_is_affine_in_the_wall_coefficients():
    prob = CylinderDrag(nr=6, nt=12, order=2, ncoef=6)
    rng = np.random.default_rng(5)
    a, b = 0.01 * rng.standard_normal(6), 0.01 * rng.standard_normal(6)
    X0 = np.asarray(prob.mesh(np.zeros(6)).nodes)
    Xa, Xb = np.asarray(prob.mesh(a).nodes), np.asarray(prob.mesh(b).nodes)
    Xab = np.asarray(prob.mesh(a + b).nodes)
    assert np.abs(Xab - (Xa + Xb - X0)).max() <= 1e-13 * np.abs(X0).max()
    # same connectivity for every coefficient set
    assert np.array_equal(np.asarray(prob.mesh(a).elements), np.asarray(prob.mesh(b).elements))
    # the wall moves radially by sum_k a_2k cos((k+1) t) + a_2k+1 sin((k+1) t);
    # the far field stays put
    r0 = np.hypot(X0[:, 0], X0[:, 1])
    wall, far = np.isclose(r0, 0.5), np.isclose(r0, 20.0)
    assert wall.sum() > 0 and far.sum() > 0
    t = np.arctan2(X0[wall, 1], X0[wall, 0])
    disp = sum(a[2 * k] * np.cos((k + 1) * t) + a[2 * k + 1] * np.sin((k + 1) * t) for k in range(3))
    ra = np.hypot(Xa[wall, 0], Xa[wall, 1])
    assert np.allclose(ra - 0.5, disp, rtol=0, atol=1e-13)
    assert np.abs(Xa[far] - X0[far]).max() <= 1e-13


def test_cylinder_mesh_generator_matches_its_description():
    m = meshgen.cylinder_omesh(4, 8, r0=0.5, r1=6.0)
    assert m.gmsh_type == 10 and np.asarray(m.elements).shape == (32, 9)
    names = sorted({f[2] for f in m.bnd_faces})
    assert names == ["FARFIELD", "WALL"]
    assert sum(1 for f in m.bnd_faces if f[2] == "WALL") == 8


def test_batched_vortex_case_parameters():
    from zefr_b200.batch import vortex_case_params
    cases = vortex_case_params(512, 4)
    assert cases == vortex_case_params(512, 4) and cases != vortex_case_params(512, 5)
    n = np.array([c["n"] for c in cases])
    P = np.array([c["P"] for c in cases])
    assert n.min() >= 8 and n.max() <= 96 and set(P.tolist()) == {1, 2, 3, 4, 5}
    for c in cases:
        assert all(-2.0 <= x <= 2.0 for x in c["center"])
        assert 1.0 <= c["beta"] <= 5.0 and 0.2 <= c["mach"] <= 0.8
        h = 10.0 / c["n"]
        want = 0.1 * h / ((c["mach"] + 1.0) * math.sqrt(1.4) * (c["P"] + 1) ** 2)
        assert c["dt"] == want
