"""Properties of the Roe flux that pin it without a reference implementation
(the reference has only Rusanov): the library's GPU Roe flux equals this
numpy restatement to 1e-12 (tests/test_gpu_parity.py), and the restatement
satisfies the defining properties of Roe's scheme (Roe 1981; Toro, Riemann
Solvers and Numerical Methods, ch. 11):

- consistency: F(U, U, n) = F(U) . n;
- conservation across the face: F(UL, UR, n) = -F(UR, UL, -n);
- Property U, seen through upwinding: with every wave speed of the Roe state
  positive (and outside the entropy-fix band) the flux is F(UL) . n exactly,
  with every one negative F(UR) . n, because |A|(UR - UL) = A (UR - UL) =
  F(UR) - F(UL) then;
- rotational invariance in 2D and 3D.
"""
import numpy as np
import pytest

from oracle.dfr_numpy import _flux_conv, _normal, roe_flux

G = 1.4


def _state(rho, vel, p):
    vel = np.asarray(vel, dtype=float)
    E = p / (G - 1.0) + 0.5 * rho * float(vel @ vel)
    return np.array([rho, *(rho * vel), E])


def _fn(U, n):
    F, _ = _flux_conv(U[:, None], G)
    return _normal(F, n[:, None])[:, 0]


def _random_pairs(D, m, seed):
    rng = np.random.default_rng(seed)
    UL = np.stack([_state(rng.uniform(0.5, 2.0), rng.uniform(-1, 1, D), rng.uniform(0.5, 2.0)) for _ in range(m)], 1)
    UR = np.stack([_state(rng.uniform(0.5, 2.0), rng.uniform(-1, 1, D), rng.uniform(0.5, 2.0)) for _ in range(m)], 1)
    n = rng.standard_normal((D, m))
    n /= np.linalg.norm(n, axis=0)
    return UL, UR, n


@pytest.mark.parametrize("D", [2, 3])
def test_consistency(D):
    UL, _, n = _random_pairs(D, 50, 1)
    F = roe_flux(UL, UL, n, G)
    for k in range(UL.shape[1]):
        assert np.allclose(F[:, k], _fn(UL[:, k], n[:, k]), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("D", [2, 3])
def test_conservation_across_the_face(D):
    UL, UR, n = _random_pairs(D, 50, 2)
    assert np.allclose(roe_flux(UL, UR, n, G), -roe_flux(UR, UL, -n, G), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("D", [2, 3])
def test_supersonic_states_are_upwinded_exactly(D):
    """Property U: all Roe-state wave speeds of one sign leave the upwind flux."""
    rng = np.random.default_rng(3)
    for k in range(40):
        n = rng.standard_normal(D)
        n /= np.linalg.norm(n)
        t = rng.standard_normal(D)
        t -= (t @ n) * n
        # Mach 3 to 4 along n, different densities, pressures, tangential speeds
        rL, rR, pL, pR = rng.uniform(0.5, 2.0, 4)
        aL, aR = np.sqrt(G * pL / rL), np.sqrt(G * pR / rR)
        for sign in (1.0, -1.0):
            UL = _state(rL, sign * rng.uniform(3, 4) * aL * n + 0.3 * t, pL)
            UR = _state(rR, sign * rng.uniform(3, 4) * aR * n - 0.2 * t, pR)
            F = roe_flux(UL[:, None], UR[:, None], n[:, None], G)[:, 0]
            up = _fn(UL, n) if sign > 0 else _fn(UR, n)
            assert np.allclose(F, up, rtol=1e-12, atol=1e-12 * np.abs(up).max())


def test_rotational_invariance_2d():
    UL, UR, n = _random_pairs(2, 30, 4)
    th = 0.7
    R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])

    def rot(U):
        out = U.copy()
        out[1:3] = R @ U[1:3]
        return out

    F = roe_flux(UL, UR, n, G)
    Fr = roe_flux(rot(UL), rot(UR), R @ n, G)
    assert np.allclose(Fr[0], F[0], rtol=1e-12, atol=1e-12)
    assert np.allclose(Fr[1:3], R @ F[1:3], rtol=1e-12, atol=1e-12)
    assert np.allclose(Fr[3], F[3], rtol=1e-12, atol=1e-12)
