"""Initial conditions of the DFR workloads, evaluated at solution points.

All functions take coordinates ``X`` of shape (S, D, E) (the reference's
``coord_spts`` layout) and return conserved variables U of shape (S, V, E).
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np


def conserved(rho, vel, p, gamma):
    """Primitive -> conserved in the reference order (rho, rho*u.., E)."""
    D = len(vel)
    out = [rho] + [rho * v for v in vel]
    ke = sum(v * v for v in vel)
    out.append(p / (gamma - 1.0) + 0.5 * rho * ke)
    return np.stack(out, axis=1)


def isentropic_vortex(X: np.ndarray, beta: float = 5.0, center=(0.0, 0.0), u_inf=(1.0, 0.0), rho_inf: float = 1.0,
                      p_inf: float = 1.0, gamma: float = 1.4) -> np.ndarray:
    """Isentropic vortex of strength beta on a uniform stream (Shu's form):
    du = -beta/(2 pi) (y-yc) e^{(1-r^2)/2}, dv = beta/(2 pi) (x-xc) e^{(1-r^2)/2},
    T = T_inf - (gamma-1) beta^2 / (8 gamma pi^2) e^{1-r^2}, isentropic p = rho^gamma scaled."""
    x = X[:, 0] - center[0]
    y = X[:, 1] - center[1]
    r2 = x * x + y * y
    e = np.exp(0.5 * (1.0 - r2))
    T_inf = p_inf / rho_inf
    T = T_inf - (gamma - 1.0) * beta ** 2 / (8.0 * gamma * math.pi ** 2) * e * e
    rho = rho_inf * (T / T_inf) ** (1.0 / (gamma - 1.0))
    p = rho * T
    u = u_inf[0] - beta / (2 * math.pi) * y * e
    v = u_inf[1] + beta / (2 * math.pi) * x * e
    return conserved(rho, [u, v], p, gamma)


def taylor_green(X: np.ndarray, mach: float = 0.1, rho0: float = 1.0, p0: float = 1.0, gamma: float = 1.4,
                 L: float = 1.0) -> np.ndarray:
    """Taylor-Green vortex (reference test_case 4, src/funcs.cpp:125-154, with
    disable_nondim so rho = p rho0 / p0 and U0 = Ma sqrt(gamma p0 / rho0))."""
    U0 = mach * math.sqrt(gamma * p0 / rho0)
    x, y, z = X[:, 0] / L, X[:, 1] / L, X[:, 2] / L
    u = U0 * np.sin(x) * np.cos(y) * np.cos(z)
    v = -U0 * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(u)
    p = p0 + rho0 * U0 * U0 / 16.0 * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0)
    rho = p * rho0 / p0
    return conserved(rho, [u, v, w], p, gamma)


def double_shear_layer(X: np.ndarray, mach: float = 0.2, delta: float = 1.0 / 30.0, eps: float = 0.05,
                       noise: float = 1e-3, seed: int = 0, gamma: float = 1.4, rho0: float = 1.0,
                       p0: float = 1.0) -> np.ndarray:
    """Doubly periodic shear layer on [0,1]^2 (Bell, Colella & Glaz 1989 form):
    u = U0 tanh((y-1/4)/delta) for y <= 1/2, U0 tanh((3/4-y)/delta) above,
    v = eps U0 sin(2 pi x), plus seeded uniform noise of relative amplitude ``noise``."""
    U0 = mach * math.sqrt(gamma * p0 / rho0)
    x, y = X[:, 0], X[:, 1]
    u = np.where(y <= 0.5, np.tanh((y - 0.25) / delta), np.tanh((0.75 - y) / delta)) * U0
    v = eps * U0 * np.sin(2 * math.pi * x)
    rng = np.random.default_rng(seed)
    u = u + noise * U0 * rng.uniform(-1, 1, size=u.shape)
    v = v + noise * U0 * rng.uniform(-1, 1, size=v.shape)
    rho = np.full_like(u, rho0)
    p = np.full_like(u, p0)
    return conserved(rho, [u, v], p, gamma)


def uniform(X: np.ndarray, rho: float, vel, p: float, gamma: float = 1.4) -> np.ndarray:
    S, D, E = X.shape
    return conserved(np.full((S, E), rho), [np.full((S, E), vel[d]) for d in range(D)], np.full((S, E), p), gamma)


def perturb(U: np.ndarray, amp: float, seed: int) -> np.ndarray:
    """Relative seeded perturbation of every conserved variable (keeps p > 0 for small amp)."""
    rng = np.random.default_rng(seed)
    scale = np.abs(U).max(axis=(0, 2), keepdims=True) + 1e-300
    return U + amp * scale * rng.uniform(-1.0, 1.0, size=U.shape)
