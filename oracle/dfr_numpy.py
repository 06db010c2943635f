"""CPU restatement of the reference DFR residual in numpy (test infrastructure).

This is the oracle the CUDA path is checked against.  It restates
``FRSolver::compute_residual`` (reference src/solver.cpp:1494-1645) step by
step on reference-layout arrays (row-major, last index fastest,
include/mdvector.hpp:189-260):

  1. U_fpts = oppE U_spts                        src/elements.cpp:1337-1360
  2. boundary ghost states                       src/faces.cpp:123-506
  3. dU_spts = oppD U_spts                       src/elements.cpp:1393-1419
     common solution (LDG)                       src/faces.cpp:1366-1474
     dU_spts += oppD_fpts Ucomm                  src/elements.cpp:1421-1447
  4. physical gradient, flux, transformed flux   src/elements.cpp:1588-1699, include/flux.hpp:1-202
  5. dU_fpts = oppE dU_spts, boundary gradient   src/elements.cpp:1362-1391, src/faces.cpp:508-710
  6. divF = oppDiv F                             src/elements.cpp:1449-1474
  7. Rusanov + LDG common flux, +-F dA           src/faces.cpp:1243-1364, 1476-1614
  8. divF += oppDiv_fpts Fcomm                   src/elements.cpp:1476-1501

The face data are organised per element flux point with the reference's
left/right roles (slot), so each face flux is evaluated identically from both
sides.  Set-up arrays come from the reference itself (golden fixtures) or from
any set-up shown equal to it.  Only tests, fixture scripts, smoke() and the
benchmark's CPU leg import this module.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Dict, Optional

import numpy as np

# reference BC_TYPE codes (include/input.hpp:54-70)
BC_CHAR, BC_SUP_IN, BC_SUP_OUT, BC_SLIP, BC_ISO, BC_ADI, BC_ISO_MOVE, BC_ADI_MOVE, BC_SYM = 2, 3, 4, 5, 6, 7, 8, 9, 11


@dataclass
class Setup:
    """Reference-layout set-up arrays of one element type."""

    ndims: int
    oppE: np.ndarray         # [Fp, S]
    oppD: np.ndarray         # [D, S, S]
    oppD_fpts: np.ndarray    # [D, S, Fp]
    oppDiv: np.ndarray       # [S, D, S]
    oppDiv_fpts: np.ndarray  # [S, Fp]
    inv_jaco: np.ndarray     # [D, S, D, E]
    jaco_det: np.ndarray     # [S, E]
    partner: np.ndarray      # [Fp, E] int: e'*Fp + f' or -1-bc
    slot: np.ndarray         # [Fp, E] 0 left / 1 right
    norm: np.ndarray         # [Fp, D, E] left unit normal
    dA: np.ndarray           # [Fp, E] own dA

    @staticmethod
    def from_arrays(ndims: int, nspts: int, nfpts: int, neles: int, get) -> "Setup":
        D, S, Fp, E = ndims, nspts, nfpts, neles
        return Setup(
            ndims=D,
            oppE=get("oppE").reshape(Fp, S), oppD=get("oppD").reshape(D, S, S),
            oppD_fpts=get("oppD_fpts").reshape(D, S, Fp), oppDiv=get("oppDiv").reshape(S, D, S),
            oppDiv_fpts=get("oppDiv_fpts").reshape(S, Fp),
            inv_jaco=get("inv_jaco_spts").reshape(D, S, D, E), jaco_det=get("jaco_det_spts").reshape(S, E),
            partner=get("fpt_partner").astype(np.int64).reshape(Fp, E), slot=get("fpt_slot").astype(np.int64).reshape(Fp, E),
            norm=get("fpt_norm").reshape(Fp, D, E), dA=get("fpt_dA").reshape(Fp, E))


def _flux_conv(U: np.ndarray, gamma: float):
    """U [V, ...] -> F [V, D, ...], P (include/flux.hpp:11-63, zero grid velocity)."""
    V = U.shape[0]
    D = V - 2
    invrho = 1.0 / U[0]
    momF = U[1] * U[1]
    for d in range(1, D):
        momF = momF + U[d + 1] * U[d + 1]
    momF = momF * invrho
    P = (gamma - 1.0) * (U[D + 1] - 0.5 * momF)
    H = (U[D + 1] + P) * invrho
    F = np.zeros((V, D) + U.shape[1:])
    for d in range(D):
        F[0, d] = U[d + 1]
        for k in range(D):
            F[k + 1, d] = U[d + 1] * U[k + 1] * invrho + (P if k == d else 0.0)
        F[D + 1, d] = U[d + 1] * H
    return F, P


def _flux_visc_add(U: np.ndarray, dU: np.ndarray, F: np.ndarray, p: Dict[str, float]) -> None:
    """F[V, D, ...] -= viscous flux (include/flux.hpp:71-202); dU [V, D, ...]."""
    V = U.shape[0]
    D = V - 2
    gamma = p["gamma"]
    invrho = 1.0 / U[0]
    vel = [U[d + 1] * invrho for d in range(D)]
    vsq = vel[0] * vel[0]
    for d in range(1, D):
        vsq = vsq + vel[d] * vel[d]
    e_int = U[D + 1] * invrho - 0.5 * vsq
    if p["fix_vis"]:
        mu = p["mu"] + 0.0 * e_int
    else:
        rt_ratio = (gamma - 1.0) * e_int / p["rt"]
        mu = p["mu"] * np.power(rt_ratio, 1.5) * (1.0 + p["c_sth"]) / (rt_ratio + p["c_sth"])
    dvel = [[(dU[i + 1, j] - dU[0, j] * vel[i]) * invrho for j in range(D)] for i in range(D)]
    de = []
    for j in range(D):
        s = vel[0] * dvel[0][j]
        for i in range(1, D):
            s = s + vel[i] * dvel[i][j]
        dke = 0.5 * vsq * dU[0, j] + U[0] * s
        de.append((dU[D + 1, j] - dke - dU[0, j] * e_int) * invrho)
    div = dvel[0][0]
    for d in range(1, D):
        div = div + dvel[d][d]
    diag = div / 3.0
    kappa = (mu / p["prandtl"]) * gamma
    for j in range(D):
        w = 0.0
        for i in range(D):
            tau = 2.0 * mu * (dvel[i][i] - diag) if i == j else mu * (dvel[i][j] + dvel[j][i])
            F[i + 1, j] -= tau
            w = w + vel[i] * tau
        F[D + 1, j] -= (w + kappa * de[j])


def _ghost(bc: np.ndarray, UL: np.ndarray, n: np.ndarray, p: Dict[str, float]):
    """Ghost (Rusanov) and prescribed (LDG) right states (src/faces.cpp:123-506).

    UL [V, M], n [D, M], bc [M] -> UR, UB [V, M]."""
    V, M = UL.shape
    D = V - 2
    g = p["gamma"]
    UR = UL.copy()
    UB = UL.copy()
    V_fs = np.array([p["V_fs0"], p["V_fs1"], p["V_fs2"]])[:D]
    V_wall = np.array([p["V_wall0"], p["V_wall1"], p["V_wall2"]])[:D]
    m = bc == BC_SUP_IN
    if m.any():
        UR[0, m] = p["rho_fs"]
        vsq = 0.0
        for d in range(D):
            UR[d + 1, m] = p["rho_fs"] * V_fs[d]
            vsq += V_fs[d] * V_fs[d]
        UR[D + 1, m] = p["P_fs"] / (g - 1.0) + 0.5 * p["rho_fs"] * vsq
        UB[:, m] = UR[:, m]
    m = bc == BC_CHAR
    if m.any():
        u = UL[:, m]
        nn = n[:, m]
        VnL = sum(u[d + 1] / u[0] * nn[d] for d in range(D))
        VnR = sum(V_fs[d] * nn[d] for d in range(D))
        momF = sum(u[d + 1] * u[d + 1] for d in range(D)) / u[0]
        PL = (g - 1.0) * (u[D + 1] - 0.5 * momF)
        PR = p["P_fs"]
        cL = np.sqrt(g * PL / u[0])
        cR = np.sqrt(g * PR / p["rho_fs"])
        sup = np.abs(VnR) >= cR
        RL = np.where(sup & (VnL >= 0), VnR + 2.0 / (g - 1) * cR, VnL + 2.0 / (g - 1) * cL)
        RB = np.where(sup & (VnL < 0), VnL - 2.0 / (g - 1) * cL, VnR - 2.0 / (g - 1) * cR)
        cstar = 0.25 * (g - 1) * (RL - RB)
        ustarn = 0.5 * (RL + RB)
        rhoR = cstar * cstar / g
        inflow = VnL < 0.0
        rhoR = rhoR * np.where(inflow, p["rho_fs"] ** g / PR, np.power(u[0], g) / PL)
        VR = [np.where(inflow, V_fs[d] + (ustarn - VnR) * nn[d], u[d + 1] / u[0] + (ustarn - VnL) * nn[d])
              for d in range(D)]
        rhoR = np.power(rhoR, 1.0 / (g - 1))
        out = np.empty_like(u)
        out[0] = rhoR
        for d in range(D):
            out[d + 1] = rhoR * VR[d]
        PRs = rhoR / g * cstar * cstar
        E = PRs / (g - 1)
        for d in range(D):
            E = E + 0.5 * rhoR * VR[d] * VR[d]
        out[D + 1] = E
        UR[:, m] = out
        UB[:, m] = out
    m = (bc == BC_SLIP) | (bc == BC_SYM)
    if m.any():
        u = UL[:, m]
        nn = n[:, m]
        momN = sum(u[d + 1] * nn[d] for d in range(D))
        for d in range(D):
            UR[d + 1, m] = u[d + 1] - 2.0 * momN * nn[d]
        UB[:, m] = UR[:, m]
    for code in (BC_ISO, BC_ISO_MOVE):
        m = bc == code
        if not m.any():
            continue
        moving = code == BC_ISO_MOVE
        u = UL[:, m]
        rhoL = u[0]
        vsq = 0.0
        vwsq = 0.0
        for d in range(D):
            vw = V_wall[d] if moving else 0.0
            V = -(u[d + 1] / rhoL) + 2 * vw
            UR[d + 1, m] = rhoL * V
            vsq = vsq + V * V
            UB[d + 1, m] = rhoL * vw if moving else vw
            vwsq += vw * vw
        cpg = p["R_ref"] / (g - 1)
        UR[D + 1, m] = rhoL * (cpg * p["T_wall"] + 0.5 * vsq)
        UB[D + 1, m] = rhoL * (cpg * p["T_wall"] + 0.5 * vwsq) if moving else rhoL * cpg * p["T_wall"]
    for code in (BC_ADI, BC_ADI_MOVE):
        m = bc == code
        if not m.any():
            continue
        moving = code == BC_ADI_MOVE
        u = UL[:, m]
        rhoL = u[0]
        vsq = 0.0
        vlsq = 0.0
        vwsq = 0.0
        for d in range(D):
            vw = V_wall[d] if moving else 0.0
            VL = u[d + 1] / rhoL
            V = -VL + 2 * vw
            UR[d + 1, m] = rhoL * V
            UB[d + 1, m] = rhoL * vw
            vsq = vsq + V * V
            vlsq = vlsq + VL * VL
            vwsq += vw * vw
        EL = u[D + 1]
        UR[D + 1, m] = EL + 0.5 * rhoL * (vsq - vlsq)
        UB[D + 1, m] = EL - 0.5 * rhoL * (vlsq + vwsq) if moving else EL + 0.5 * rhoL * (vwsq - vlsq)
    return UR, UB


def _ghost_grad(bc: np.ndarray, UL: np.ndarray, dUL: np.ndarray, n: np.ndarray) -> np.ndarray:
    """Right-state gradient on boundaries (src/faces.cpp:508-710). dUL [V, D, M]."""
    dUR = dUL.copy()
    V = UL.shape[0]
    D = V - 2
    m = (bc == BC_ADI) | (bc == BC_ADI_MOVE)
    if m.any():
        u = UL[:, m]
        du = dUL[:, :, m]
        nn = n[:, m]
        rho, E = u[0], u[D + 1]
        vel = [u[d + 1] / rho for d in range(D)]
        dTn = 0.0
        for j in range(D):
            s = 0.0
            for i in range(D):
                s = s + vel[i] * ((du[i + 1, j] - du[0, j] * vel[i]) / rho)
            dT = du[D + 1, j] - du[0, j] * E / rho - rho * s
            dTn = dTn + dT * nn[j]
        for j in range(D):
            dUR[D + 1, j, m] = du[D + 1, j] - dTn * nn[j]
    return dUR


def _normal(F: np.ndarray, n: np.ndarray) -> np.ndarray:
    """F [V, D, M], n [D, M] -> F.n [V, M] (sum in dimension order)."""
    out = F[:, 0] * n[0]
    for d in range(1, n.shape[0]):
        out = out + F[:, d] * n[d]
    return out


def roe_flux(UL: np.ndarray, UR: np.ndarray, n: np.ndarray, gamma: float) -> np.ndarray:
    """Roe approximate Riemann flux (Roe 1981; eigen-decomposition as in Toro,
    Riemann Solvers and Numerical Methods, sec. 11.3) with Harten's entropy fix
    (|l| < delta -> (l^2 + delta^2)/(2 delta), delta = 0.1 (|u_n| + a) of the
    Roe state).  No reference counterpart: the reference has only Rusanov.
    UL, UR [V, M]; n [D, M] unit normals."""
    V = UL.shape[0]
    D = V - 2
    FL, PL = _flux_conv(UL, gamma)
    FR, PR = _flux_conv(UR, gamma)
    rL, rR = UL[0], UR[0]
    sL, sR = np.sqrt(rL), np.sqrt(rR)
    inv = 1.0 / (sL + sR)
    uL = [UL[d + 1] / rL for d in range(D)]
    uR = [UR[d + 1] / rR for d in range(D)]
    u = [(sL * uL[d] + sR * uR[d]) * inv for d in range(D)]
    unL = sum(uL[d] * n[d] for d in range(D))
    unR = sum(uR[d] * n[d] for d in range(D))
    H = (sL * (UL[D + 1] + PL) / rL + sR * (UR[D + 1] + PR) / rR) * inv
    q2 = sum(u[d] * u[d] for d in range(D))
    un = sum(u[d] * n[d] for d in range(D))
    a2 = np.maximum((gamma - 1.0) * (H - 0.5 * q2), 1e-30)
    a = np.sqrt(a2)
    rho = sL * sR
    dp, dr, dun = PR - PL, rR - rL, unR - unL
    a1 = (dp - rho * a * dun) / (2.0 * a2)
    a3 = (dp + rho * a * dun) / (2.0 * a2)
    a2w = dr - dp / a2
    delta = 0.1 * (np.abs(un) + a)

    def fix(lam):
        lam = np.abs(lam)
        return np.where(lam < delta, (lam * lam + delta * delta) / (2.0 * delta), lam)

    l1, l2, l3 = fix(un - a), fix(un), fix(un + a)
    dvt = [(uR[d] - uL[d]) - dun * n[d] for d in range(D)]
    diss = np.empty_like(UL)
    diss[0] = l1 * a1 + l2 * a2w + l3 * a3
    for d in range(D):
        diss[d + 1] = l1 * a1 * (u[d] - a * n[d]) + l2 * (a2w * u[d] + rho * dvt[d]) + l3 * a3 * (u[d] + a * n[d])
    udvt = sum(u[d] * dvt[d] for d in range(D))
    diss[D + 1] = l1 * a1 * (H - a * un) + l2 * (a2w * 0.5 * q2 + rho * udvt) + l3 * a3 * (H + a * un)
    return 0.5 * (_normal(FL, n) + _normal(FR, n)) - 0.5 * diss


def residual(st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool, fconv: str = "rusanov") -> np.ndarray:
    """divF_spts(stage) for state U [S, V, E] (reference form, |J| div F).

    fconv "rusanov" restates the reference; "roe" swaps in :func:`roe_flux`."""
    if fconv not in ("rusanov", "roe"):
        raise ValueError("unknown convective flux " + fconv)
    S, V, E = U.shape
    D = st.ndims
    Fp = st.oppE.shape[0]
    gamma = p["gamma"]
    # 1. extrapolate
    Ufp = np.einsum("fs,sve->fve", st.oppE, U)
    # per element fpt: own and partner states, flattened over (f, e)
    own = Ufp.transpose(1, 0, 2).reshape(V, Fp * E)                    # [V, Fp*E] index f*E+e
    part = st.partner.reshape(-1)
    interior = part >= 0
    pe = np.where(interior, part // Fp, 0)
    pf = np.where(interior, part % Fp, 0)
    other = Ufp[pf, :, pe].T                                            # [V, M]
    slot = st.slot.reshape(-1)
    n = st.norm.transpose(1, 0, 2).reshape(D, Fp * E)
    dA = st.dA.reshape(-1)
    bc = np.where(interior, 0, -1 - part)
    UL = np.where(slot == 0, own, other)
    URi = np.where(slot == 0, other, own)
    URg, UBg = _ghost(bc, own, n, p)
    UR = np.where(interior, URi, URg)   # Rusanov right state
    UB = np.where(interior, URi, UBg)   # LDG right state
    inv = st.inv_jaco  # [D1, S, D2, E]
    det = st.jaco_det
    dU_phys = None
    beta = p["ldg_b"]
    if viscous:
        # 3. corrected gradient
        dU = np.einsum("dst,tve->dsve", st.oppD, U)
        if beta == 0.5:
            UC = UB.copy()
        elif beta == -0.5:
            UC = UL.copy()
        else:
            UC = 0.5 * (UL + UB) - beta * (UL - UB)
        UC = np.where(interior, UC, UBg)
        Ucomm = UC.reshape(V, Fp, E).transpose(1, 0, 2)
        dU = dU + np.einsum("dsf,fve->dsve", st.oppD_fpts, Ucomm)
        # physical gradient dU[d1] = sum_d2 tdU[d2] inv[d2][d1] / |J|
        dU_phys = np.zeros_like(dU)
        for d1 in range(D):
            acc = 0.0
            for d2 in range(D):
                acc = acc + dU[d2] * inv[d2, :, d1][:, None, :]
            dU_phys[d1] = acc * (1.0 / det)[:, None, :]
    # 4. flux at solution points
    Uv = U.transpose(1, 0, 2)                                           # [V, S, E]
    F, _ = _flux_conv(Uv, gamma)                                        # [V, D, S, E]
    if viscous:
        _flux_visc_add(Uv, dU_phys.transpose(2, 0, 1, 3), F, p)        # dU as [V, D, S, E]
    Ft = np.zeros((D, S, V, E))
    for d1 in range(D):
        acc = 0.0
        for d2 in range(D):
            acc = acc + F[:, d2] * inv[d1, :, d2][None, :, :]
        Ft[d1] = acc.transpose(1, 0, 2)
    # 6. volume divergence
    divF = np.einsum("sdt,dtve->sve", st.oppDiv, Ft)
    # 7. common flux
    FL, PL = _flux_conv(UL, gamma)
    FR, PR = _flux_conv(UR, gamma)
    aL = np.sqrt(gamma * PL / UL[0])
    aR = np.sqrt(gamma * PR / UR[0])
    VnL = sum(UL[d + 1] / UL[0] * n[d] for d in range(D))
    VnR = sum(UR[d + 1] / UR[0] * n[d] for d in range(D))
    eig = np.maximum(np.abs(VnL) + aL, np.abs(VnR) + aR)
    if fconv == "roe":
        Fc = roe_flux(UL, UR, n, gamma)
    else:
        Fc = 0.5 * (_normal(FR, n) + _normal(FL, n)) - 0.5 * eig * (1.0 - p["rus_k"]) * (UR - UL)
    sign = np.where(slot == 0, 1.0, -1.0)
    Fcomm = sign * Fc * dA
    if viscous:
        dUf = np.einsum("fs,dsve->vdfe", st.oppE, dU_phys).reshape(V, D, Fp * E)
        dUo = dUf
        dUp = dUf.reshape(V, D, Fp, E)[:, :, pf, pe]
        dUL = np.where(slot == 0, dUo, dUp)
        dUR = np.where(slot == 0, dUp, dUo)
        dURg = _ghost_grad(bc, own, dUo, n)
        dUR = np.where(interior, dUR, dURg)
        ULv = UL
        URv = UB
        tau = p["ldg_tau"]
        if beta == 0.5:
            dUR = np.where(interior, 0.0, dUR)
        elif beta == -0.5:
            dUL = np.where(interior, 0.0, dUL)
        FvL = np.zeros((V, D, Fp * E))
        FvR = np.zeros((V, D, Fp * E))
        _flux_visc_add(ULv, dUL, FvL, p)
        _flux_visc_add(URv, dUR, FvR, p)
        FnL = _normal(FvL, n)
        FnR = _normal(FvR, n)
        Fv_int = 0.5 * (FnL + FnR) + tau * (ULv - URv) + beta * (FnL - FnR)
        Fv_bnd = FnR + tau * (ULv - URv)
        Fv = np.where(interior, Fv_int, Fv_bnd)
        Fcomm = Fcomm + sign * Fv * dA
    Fcomm = Fcomm.reshape(V, Fp, E).transpose(1, 0, 2)
    # 8. surface correction
    return divF + np.einsum("sf,fve->sve", st.oppDiv_fpts, Fcomm)


def physical_gradient(st: Setup, U: np.ndarray, p: Dict[str, float]) -> np.ndarray:
    """LDG-corrected physical gradient [D, S, V, E] of compute_dU_spts/_fpts +
    compute_F (src/elements.cpp:1393-1447, 1620-1653)."""
    S, V, E = U.shape
    D = st.ndims
    Fp = st.oppE.shape[0]
    Ufp = np.einsum("fs,sve->fve", st.oppE, U)
    own = Ufp.transpose(1, 0, 2).reshape(V, Fp * E)
    part = st.partner.reshape(-1)
    interior = part >= 0
    pe = np.where(interior, part // Fp, 0)
    pf = np.where(interior, part % Fp, 0)
    other = Ufp[pf, :, pe].T
    slot = st.slot.reshape(-1)
    n = st.norm.transpose(1, 0, 2).reshape(D, Fp * E)
    bc = np.where(interior, 0, -1 - part)
    UL = np.where(slot == 0, own, other)
    URi = np.where(slot == 0, other, own)
    _, UBg = _ghost(bc, own, n, p)
    UB = np.where(interior, URi, UBg)
    beta = p["ldg_b"]
    if beta == 0.5:
        UC = UB.copy()
    elif beta == -0.5:
        UC = UL.copy()
    else:
        UC = 0.5 * (UL + UB) - beta * (UL - UB)
    UC = np.where(interior, UC, UBg)
    Ucomm = UC.reshape(V, Fp, E).transpose(1, 0, 2)
    dU = np.einsum("dst,tve->dsve", st.oppD, U) + np.einsum("dsf,fve->dsve", st.oppD_fpts, Ucomm)
    out = np.zeros_like(dU)
    for d1 in range(D):
        acc = 0.0
        for d2 in range(D):
            acc = acc + dU[d2] * st.inv_jaco[d2, :, d1][:, None, :]
        out[d1] = acc * (1.0 / st.jaco_det)[:, None, :]
    return out


def functionals(st: Setup, U: np.ndarray, weights: np.ndarray, p: Dict[str, float], viscous: bool):
    """Kinetic energy, enstrophy and volume integrals (report_turbulent_stats,
    src/solver.cpp:7813-7917), unnormalised."""
    S, V, E = U.shape
    D = st.ndims
    jw = st.jaco_det * weights[:, None]
    rho = U[:, 0]
    vel = [U[:, d + 1] / rho for d in range(D)]
    ke = float((jw * 0.5 * rho * sum(v * v for v in vel)).sum())
    en = 0.0
    if viscous:
        g = physical_gradient(st, U, p)  # [D, S, V, E]
        du = [[(g[j, :, i + 1] - g[j, :, 0] * vel[i]) / rho for j in range(D)] for i in range(D)]
        if D == 3:
            w2 = (du[2][1] - du[1][2]) ** 2 + (du[0][2] - du[2][0]) ** 2 + (du[1][0] - du[0][1]) ** 2
        else:
            w2 = (du[1][0] - du[0][1]) ** 2
        en = float((jw * 0.5 * rho * w2).sum())
    return {"ke": ke, "enstrophy": en, "volume": float(jw.sum())}


WALL_BCS = (BC_SLIP, BC_ISO, BC_ADI, BC_ISO_MOVE, BC_ADI_MOVE)


def wall_force(st: Setup, U: np.ndarray, wfpt: np.ndarray, coord_fpts: np.ndarray, p: Dict[str, float],
               viscous: bool):
    """Force and moment (about the origin) on wall boundaries of
    FRSolver::compute_moments (src/solver.cpp:7600-7811): per wall flux point
    w * (P n - tau n) * dA from the element's own trace and its extrapolated
    corrected gradient.  In 3D the reference reads the state of flux point 0
    for the viscous stress (src/solver.cpp:7716-7720); this restatement uses
    each flux point's own state.  wfpt [Fp] face quadrature weights,
    coord_fpts [Fp, D, E]."""
    S, V, E = U.shape
    D = st.ndims
    g = p["gamma"]
    Ufp = np.einsum("fs,sve->fve", st.oppE, U)
    bc = np.where(st.partner < 0, -1 - st.partner, 0)
    wall = np.isin(bc, WALL_BCS)
    rho = Ufp[:, 0]
    vel = [Ufp[:, d + 1] / rho for d in range(D)]
    P = (g - 1.0) * (Ufp[:, D + 1] - 0.5 * rho * sum(v * v for v in vel))
    w = wfpt[:, None] * st.dA
    force = np.zeros(3)
    moment = np.zeros(3)
    fx = np.zeros((3,) + P.shape)
    for d in range(D):
        fx[d] = w * P * st.norm[:, d]
    if viscous:
        dUs = physical_gradient(st, U, p)                     # [D, S, V, E]
        dUf = np.einsum("fs,dsve->dfve", st.oppE, dUs)         # [D, Fp, V, E]
        if p["fix_vis"]:
            mu = np.full_like(rho, p["mu"])
        else:
            e_int = Ufp[:, D + 1] / rho - 0.5 * sum(v * v for v in vel)
            rt = (g - 1.0) * e_int / p["rt"]
            mu = p["mu"] * rt ** 1.5 * (1.0 + p["c_sth"]) / (rt + p["c_sth"])
        gv = [[(dUf[j, :, i + 1] - dUf[j, :, 0] * vel[i]) / rho for j in range(D)] for i in range(D)]
        diag = sum(gv[i][i] for i in range(D)) / 3.0
        tau = [[None] * D for _ in range(D)]
        for i in range(D):
            for j in range(D):
                tau[i][j] = 2.0 * mu * (gv[i][i] - diag) if i == j else mu * (gv[i][j] + gv[j][i])
        for i in range(D):
            taun = sum(tau[i][j] * st.norm[:, j] for j in range(D))
            fx[i] = fx[i] - w * taun
    for d in range(D):
        force[d] = float(fx[d][wall].sum())
    x = coord_fpts[:, 0]
    y = coord_fpts[:, 1]
    if D == 2:
        moment[2] = float((x * fx[1] - y * fx[0])[wall].sum())
    else:
        z = coord_fpts[:, 2]
        moment[0] = float((y * fx[2] - z * fx[1])[wall].sum())
        moment[1] = float((z * fx[0] - x * fx[2])[wall].sum())
        moment[2] = float((x * fx[1] - y * fx[0])[wall].sum())
    return force, moment


def rk44_step(st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool, dt: float) -> np.ndarray:
    """One explicit RK44 step (FRSolver::step_RK, src/solver.cpp:2864-3097)."""
    alpha = [0.5, 0.5, 1.0]
    beta = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]
    U_ini = U.copy()
    det = st.jaco_det[:, None, :]
    regs = []
    Us = U
    for s in range(3):
        r = residual(st, Us, p, viscous)
        regs.append(r)
        Us = U_ini - alpha[s] * dt / det * r
    regs.append(residual(st, Us, p, viscous))
    Un = U_ini.copy()
    for s in range(4):
        Un = Un - beta[s] * dt / det * regs[s]
    return Un


# ---------------------------------------------------------------------------
# time integration: RK54 (step_LSRK + step_adaptive) and the CFL time step
# (compute_element_dt); src/solver.cpp:749-777, 2663-2757, 3100-3255, 4105-4272
# ---------------------------------------------------------------------------

# Kennedy-Carpenter RK54 2N pair as tabulated in src/solver.cpp:749-777
LSRK_A = [970286171893. / 4311952581923., 6584761158862. / 12103376702013.,
          2251764453980. / 15575788980749., 26877169314380. / 34165994151039.]
LSRK_B = [1153189308089. / 22510343858157., 1772645290293. / 4653164025191.,
          -1672844663538. / 4480602732383., 2114624349019. / 3568978502595.,
          5198255086312. / 14908931495163.]
LSRK_BHAT = [1016888040809. / 7410784769900., 11231460423587. / 58533540763752.,
             -1563879915014. / 6823010717585., 606302364029. / 971179775848.,
             1097981568119. / 3980877426909.]
# get_cfl_limit_adv / get_cfl_limit_diff (src/funcs.cpp:435-560), orders 0..10
CFL_ADV = [1.392, 0.4642, 0.2351, 0.1453, 0.1000, 0.07363, 0.05678, 0.04530, 0.03709, 0.03101, 0.02635]
CFL_DIFF_CENTRED = [2.785, 0.1740, 0.04264, 0.01580, 0.007193, 0.003730, 0.002120, 0.001292, 0.0008314,
                    0.0005586, 0.0003890]
CFL_DIFF_UPWIND = [0.6963, 0.07736, 0.01878, 0.006345, 0.002664, 0.001299, 0.0007060, 0.0004153, 0.0002599,
                   0.0001708, 0.0001168]


def lsrk_step(st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool, dt: float, adapt: bool = False):
    """One RK54 step (FRSolver::step_LSRK, src/solver.cpp:3100-3255).

    Returns (U_new, rk_err); rk_err is None unless ``adapt``."""
    det = st.jaco_det[:, None, :]
    U_til = U.copy()
    Us = U.copy()
    err = np.zeros_like(U) if adapt else None
    for s in range(5):
        r = residual(st, Us, p, viscous)
        if adapt:
            err = err - (LSRK_B[s] - LSRK_BHAT[s]) * dt / det * r
        if s < 4:
            Us = U_til - LSRK_A[s] * dt / det * r
            U_til = Us - (LSRK_B[s] - LSRK_A[s]) * dt / det * r
        else:
            Us = U_til - LSRK_B[s] * dt / det * r
    return Us, err


def rk_error(U: np.ndarray, U_ini: np.ndarray, err: np.ndarray, atol: float, rtol: float) -> float:
    """Infinity norm of the scaled RK error (src/solver.cpp:2671-2684); NaN counts as infinite."""
    x = np.abs(err) / (atol + rtol * np.maximum(np.abs(U), np.abs(U_ini)))
    x = np.where(np.isnan(x), np.inf, x)
    return float(x.max())


class AdaptiveRK54:
    """step_adaptive (src/solver.cpp:2663-2757) around :func:`lsrk_step`."""

    def __init__(self, dt: float, atol=1e-5, rtol=1e-5, pi_alpha=0.7, pi_beta=0.4, safety=0.8, max_factor=2.5,
                 min_factor=0.3, max_dt=100.0):
        self.dt, self.atol, self.rtol = dt, atol, rtol
        self.expa, self.expb = pi_alpha / 4.0, pi_beta / 4.0
        self.safety, self.max_factor, self.min_factor, self.max_dt = safety, max_factor, min_factor, max_dt
        self.prev_err, self.rejected = 1.0, 0

    def step(self, st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool) -> np.ndarray:
        while True:
            Un, err = lsrk_step(st, U, p, viscous, self.dt, adapt=True)
            max_err = rk_error(Un, U, err, self.atol, self.rtol)
            with np.errstate(divide="ignore"):
                fac = max_err ** -self.expa * self.prev_err ** self.expb
            fac = min(self.max_factor, max(self.min_factor, self.safety * fac))
            self.dt = min(self.dt * fac, self.max_dt)
            if self.dt < 1e-14:
                raise RuntimeError("dt approaching 0")
            if max_err < 1.0:
                self.prev_err = max_err
                return Un
            self.rejected += 1


def h_ref(coord_fpts: np.ndarray, loc_fpts: np.ndarray, nfpts_face: int) -> np.ndarray:
    """Tensor-line lengths between paired flux points of opposite faces
    (src/elements.cpp:408-483) from coord_fpts [Fp, D, E] and loc_fpts [Fp, D].

    2D pairs point i of faces 0/1 with point N-1-i of faces 2/3; 3D sorts the
    reference positions of each face of a pair (btm/top, left/right,
    front/back) and pairs equal ranks, with the reference's length expression
    sqrt(dx^2 + dy^2 * dz^2)."""
    Fp, D, E = coord_fpts.shape
    h = np.zeros((Fp, E))
    if D == 2:
        N = nfpts_face
        for f1 in range(Fp // 2):
            i = f1 % N
            f2 = (f1 // N + 3) * N - i - 1
            d = coord_fpts[f1] - coord_fpts[f2]
            h[f1] = h[f2] = np.sqrt(d[0] * d[0] + d[1] * d[1])
        return h
    nf = nfpts_face

    def order(idx):
        pts = np.round(loc_fpts[idx], 10)
        return [idx[k] for k in np.lexsort(pts.T[::-1])]

    for f in range(3):
        a = order(np.arange(2 * f * nf, (2 * f + 1) * nf))
        b = order(np.arange((2 * f + 1) * nf, (2 * f + 2) * nf))
        for f1, f2 in zip(a, b):
            d = coord_fpts[f1] - coord_fpts[f2]
            h[f1] = h[f2] = np.sqrt(d[0] * d[0] + d[1] * d[1] * d[2] * d[2])
    return h


def element_dt(st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool, order: int, cfl: float, cfl_type: int,
               vol: np.ndarray, wfpts: np.ndarray, href: Optional[np.ndarray] = None) -> np.ndarray:
    """Per-element CFL time step of compute_element_dt (src/solver.cpp:4105-4199)
    with the face wave speed of the Rusanov flux (src/faces.cpp:1296-1316) and
    the LDG diffusion coefficient (src/faces.cpp:1572-1577) at the state U."""
    S, V, E = U.shape
    D = st.ndims
    Fp = st.oppE.shape[0]
    nf = Fp // (2 * D)
    g = p["gamma"]
    Ufp = np.einsum("fs,sve->fve", st.oppE, U)
    own = Ufp.transpose(1, 0, 2).reshape(V, Fp * E)
    part = st.partner.reshape(-1)
    interior = part >= 0
    other = Ufp[np.where(interior, part % Fp, 0), :, np.where(interior, part // Fp, 0)].T
    n = st.norm.transpose(1, 0, 2).reshape(D, Fp * E)
    bc = np.where(interior, 0, -1 - part)
    URg, UBg = _ghost(bc, own, n, p)
    UR = np.where(interior, other, URg)
    UB = np.where(interior, other, UBg)

    def ws(Uq):
        P = (g - 1.0) * (Uq[D + 1] - 0.5 * (Uq[1:D + 1] ** 2).sum(0) / Uq[0])
        a = np.sqrt(g * P / Uq[0])
        Vn = sum(Uq[d + 1] / Uq[0] * n[d] for d in range(D))
        return np.abs(Vn) + a

    wsp = np.maximum(ws(own), ws(UR)).reshape(Fp, E)
    c_adv = CFL_ADV[order]
    if cfl_type == 1:
        w = np.array([wfpts[f % nf] for f in range(Fp)])
        return 2.0 * cfl * c_adv * vol / (w[:, None] * wsp * st.dA).sum(0)
    t = wsp / (c_adv * href)
    if viscous:
        c_diff = (CFL_DIFF_CENTRED if p["ldg_b"] == 0.0 else CFL_DIFF_UPWIND)[order]
        mu, pr = p["mu"], p["prandtl"]

        def dc(rho):
            return np.maximum(mu / rho, g * mu / (pr * rho))

        t = t + np.maximum(dc(own[0]), dc(UB[0])).reshape(Fp, E) / (c_diff * href * href)
    dtinv = t.reshape(2 * D, nf, E).max(1)
    if D == 2:
        return cfl / (np.maximum(dtinv[0], dtinv[2]) + np.maximum(dtinv[1], dtinv[3]))
    return cfl / (np.maximum(dtinv[0], dtinv[1]) + np.maximum(dtinv[2], dtinv[3]) + np.maximum(dtinv[4], dtinv[5]))


def rk44_step_dt(st: Setup, U: np.ndarray, p: Dict[str, float], viscous: bool, dt) -> np.ndarray:
    """RK44 step with a global (scalar) or per-element ([E]) time step."""
    alpha = [0.5, 0.5, 1.0]
    beta = [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]
    dt = np.asarray(dt, dtype=np.float64)
    U_ini = U.copy()
    det = st.jaco_det[:, None, :]
    regs, Us = [], U
    for s in range(3):
        r = residual(st, Us, p, viscous)
        regs.append(r)
        Us = U_ini - alpha[s] * dt / det * r
    regs.append(residual(st, Us, p, viscous))
    Un = U_ini.copy()
    for s in range(4):
        Un = Un - beta[s] * dt / det * regs[s]
    return Un
