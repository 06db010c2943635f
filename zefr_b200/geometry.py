"""Differentiable geometry and wall force for shape and flow-angle gradients.

``GeometryMap`` gives the set-up metrics the residual is built on
(reference src/elements.cpp:325-407, 845-996) as differentiable functions of
the mesh node coordinates: the adjugate and |J| at solution points, and the
unit normal and area factor at flux points (the left element's normal for
both sides of a face), computed by the library's geometry kernels
(``zb_geometry_eval``, equal to the set-up bit for bit) with their adjoint
(``zb_geometry_eval_vjp``).  ``zb_vjp_geometry`` returns the residual's
adjoint with respect to exactly these arrays, so the chain rule to the nodes
is one torch backward through ``GeometryMap.metrics``.

``WallForce`` is FRSolver::compute_moments (src/solver.cpp:7600-7811) as a
torch function of the state and the metrics (the library's FP64 device
reduction ``zb_wall_force`` computes the same value; this form is what the
objective's own gradient is taken from).
"""
from __future__ import annotations

from typing import Dict

import numpy as np
import torch

WALL_BCS = (5, 6, 7, 8, 9)


def _t(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


KEYS = ("inv_jaco", "jaco_det", "norm", "dA")


class _Metrics(torch.autograd.Function):
    """Element nodes [nNodes,D,E] -> the four metric arrays by the library's
    geometry kernels (zb_geometry_eval); backward is zb_geometry_eval_vjp."""

    @staticmethod
    def forward(ctx, nodes: torch.Tensor, solver):
        out = solver.geometry_eval(nodes)
        ctx.solver = solver
        ctx.save_for_backward(nodes)
        return tuple(out[k] for k in KEYS)

    @staticmethod
    def backward(ctx, *grads):
        (nodes,) = ctx.saved_tensors
        bars = {k: g for k, g in zip(KEYS, grads) if g is not None}
        return ctx.solver.geometry_eval_vjp(nodes, bars), None


class GeometryMap:
    """Set-up metrics of a solver's mesh as differentiable functions of the
    mesh node coordinates X [n_nodes, D]: element nodes gathered in torch,
    metrics and their adjoint by the library's geometry kernels."""

    def __init__(self, solver, mesh, device="cuda"):
        D = solver.ndims
        self.s = solver
        self.D, self.S, self.E, self.Fp = D, solver.nspts, solver.neles, solver.info.nfpts
        self.dev = device
        self.e2n = torch.as_tensor(np.asarray(mesh.elements, dtype=np.int64), device=device)
        self.nodes0 = _t(np.asarray(mesh.nodes)[:, :D], device)

    def element_nodes(self, X: torch.Tensor) -> torch.Tensor:
        """X [n_nodes, D] -> element nodes [nNodes, D, E] (Elements::nodes)."""
        return X[self.e2n].permute(1, 2, 0).contiguous()

    def metrics(self, X: torch.Tensor) -> Dict[str, torch.Tensor]:
        """X [n_nodes, D] -> inv_jaco [D,S,D,E], jaco_det [S,E], norm [Fp,D,E], dA [Fp,E]."""
        return dict(zip(KEYS, _Metrics.apply(self.element_nodes(X), self.s)))


class WallForce:
    """compute_moments' force on the wall boundaries as a torch function of the
    state U [S,V,E] and the metrics (2D and 3D; each flux point's own state)."""

    def __init__(self, solver, params: Dict[str, float], device="cuda"):
        p = solver.plan
        D, S, E, Fp = solver.ndims, solver.nspts, solver.neles, solver.info.nfpts
        self.D, self.S, self.E, self.Fp = D, S, E, Fp
        self.p = params
        self.oppE = _t(p.get("oppE").reshape(Fp, S), device)
        self.oppD = _t(p.get("oppD").reshape(D, S, S), device)
        self.oppDf = _t(p.get("oppD_fpts").reshape(D, S, Fp), device)
        part = p.get("fpt_partner").reshape(Fp, E).astype(np.int64)
        slot = p.get("fpt_slot").reshape(Fp, E).astype(np.int64)
        bc = np.where(part < 0, -1 - part, 0)
        wall = np.isin(bc, WALL_BCS)
        self.W = np.where(wall.any(axis=0))[0]                 # wall elements
        self.wall = torch.as_tensor(wall[:, self.W], device=device)
        N = solver.info.order + 1
        w1 = np.polynomial.legendre.leggauss(N)[1]
        if D == 3:
            fw = np.array([w1[(f % (N * N)) // N] * w1[(f % (N * N)) % N] for f in range(Fp)])
        else:
            fw = np.array([w1[f % N] for f in range(Fp)])
        self.fw = _t(fw, device)
        interior = part >= 0
        self.interior = torch.as_tensor(interior[:, self.W], device=device)
        self.slot = torch.as_tensor(slot[:, self.W], device=device)
        self.pe = torch.as_tensor(np.where(interior, part // Fp, 0)[:, self.W], device=device)
        self.pf = torch.as_tensor(np.where(interior, part % Fp, 0)[:, self.W], device=device)
        self.bc = torch.as_tensor(bc[:, self.W], device=device)
        self.Wt = torch.as_tensor(self.W, device=device)
        if not params.get("viscous", 1.0):
            self.viscous = False
        else:
            self.viscous = True

    def _wall_state(self, U: torch.Tensor, bc: torch.Tensor, n: torch.Tensor) -> torch.Tensor:
        """LDG boundary state UB of the wall conditions (src/faces.cpp:123-506)
        for traces U [V, ...]; other boundary codes keep the trace."""
        D = self.D
        g = self.p["gamma"]
        rho = U[0]
        vel = [U[d + 1] / rho for d in range(D)]
        vlsq = sum(v * v for v in vel)
        out = [rho]
        iso = (bc == 6)
        adi = (bc == 7)
        slip = (bc == 5) | (bc == 11)
        momN = sum(U[d + 1] * n[d] for d in range(D))
        for d in range(D):
            m = U[d + 1]
            m = torch.where(iso | adi, torch.zeros_like(m), m)
            m = torch.where(slip, U[d + 1] - 2.0 * momN * n[d], m)
            out.append(m)
        E = U[D + 1]
        cpg = self.p["R_ref"] / (g - 1.0)
        E = torch.where(adi, U[D + 1] - 0.5 * rho * vlsq, E)
        E = torch.where(iso, rho * cpg * self.p["T_wall"], E)
        out.append(E)
        return torch.stack(out, dim=0)

    def force(self, U: torch.Tensor, geo: Dict[str, torch.Tensor]) -> torch.Tensor:
        D, S, Fp = self.D, self.S, self.Fp
        g = self.p["gamma"]
        V = D + 2
        W = self.Wt
        Ufp_all = torch.einsum("fs,sve->fve", self.oppE, U)          # [Fp, V, E]
        Uw = U[:, :, W]
        Ufp = Ufp_all[:, :, W]                                       # [Fp, V, Ew]
        n = geo["norm"][:, :, W]                                     # [Fp, D, Ew]
        dA = geo["dA"][:, W]
        rho = Ufp[:, 0]
        vel = [Ufp[:, d + 1] / rho for d in range(D)]
        P = (g - 1.0) * (Ufp[:, D + 1] - 0.5 * rho * sum(v * v for v in vel))
        wdA = self.fw[:, None] * dA
        F = [wdA * P * n[:, d] for d in range(D)]
        if self.viscous:
            # LDG common solution at the wall elements' flux points
            other = Ufp_all[self.pf, :, self.pe]                      # [Fp, Ew, V]
            other = other.permute(0, 2, 1)
            beta = self.p["ldg_b"]
            slot = self.slot[:, None, :]
            UL = torch.where(slot == 0, Ufp, other)
            UR = torch.where(slot == 0, other, Ufp)
            UCi = (0.5 - beta) * UL + (0.5 + beta) * UR
            UB = self._wall_state(Ufp.permute(1, 0, 2), self.bc, n.permute(1, 0, 2)).permute(1, 0, 2)
            UC = torch.where(self.interior[:, None, :], UCi, UB)
            tdU = torch.einsum("dst,tve->dsve", self.oppD, Uw) + torch.einsum("dsf,fve->dsve", self.oppDf, UC)
            inv = geo["inv_jaco"][:, :, :, W]
            det = geo["jaco_det"][:, W]
            dU = torch.stack([sum(tdU[d2] * inv[d2, :, d1][:, None, :] for d2 in range(D)) / det[:, None, :]
                              for d1 in range(D)], dim=0)            # [D, S, V, Ew]
            dUf = torch.einsum("fs,dsve->dfve", self.oppE, dU)       # [D, Fp, V, Ew]
            if self.p["fix_vis"]:
                mu = self.p["mu"]
            else:
                e_int = Ufp[:, D + 1] / rho - 0.5 * sum(v * v for v in vel)
                rr = (g - 1.0) * e_int / self.p["rt"]
                mu = self.p["mu"] * rr ** 1.5 * (1.0 + self.p["c_sth"]) / (rr + self.p["c_sth"])
            gv = [[(dUf[j, :, i + 1] - dUf[j, :, 0] * vel[i]) / rho for j in range(D)] for i in range(D)]
            diag = sum(gv[i][i] for i in range(D)) / 3.0
            for i in range(D):
                taun = 0.0
                for j in range(D):
                    tau = 2.0 * mu * (gv[i][i] - diag) if i == j else mu * (gv[i][j] + gv[j][i])
                    taun = taun + tau * n[:, j]
                F[i] = F[i] - wdA * taun
        wall = self.wall
        return torch.stack([torch.where(wall, F[d], torch.zeros_like(F[d])).sum() for d in range(D)])
