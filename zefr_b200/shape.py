"""Adjoint of the laminar cylinder: time-averaged drag over RK44 steps,
differentiated with respect to Fourier wall-displacement coefficients and
the free-stream angle.

The mesh is ``meshgen.cylinder_omesh`` (9-node quads, radial stretching) with
its wall displaced radially by sum_k a_{2k} cos((k+1) t) + a_{2k+1} sin((k+1) t),
the displacement decaying linearly to zero at the far field, so the node
coordinates are linear in the coefficients.  The flow starts from the
uniform free stream at angle alpha (characteristic far field, adiabatic
no-slip wall).  The objective is the mean over the steps of the wall force
(FRSolver::compute_moments, src/solver.cpp:7600-7811) along the free-stream
direction.

Gradient: the checkpointed trajectory adjoint (``autograd.TrajectoryAdjoint``)
gives dJ/dU0, dJ/d(free stream) and dJ/d(metrics) through the library's
hand-written adjoint (``zb_vjp_geometry``); the metrics' dependence on the
nodes is ``geometry.GeometryMap`` under torch autograd.
"""
from __future__ import annotations

import math
from typing import Dict, Sequence

import numpy as np
import torch

from . import ics, meshgen
from .autograd import TrajectoryAdjoint
from .geometry import GeometryMap, WallForce
from .solver import FRSolver, make_params


class CylinderDrag:
    def __init__(self, nr: int = 48, nt: int = 96, order: int = 3, mach: float = 0.2, reynolds: float = 100.0,
                 r1: float = 20.0, stretch: float = 1.1, ncoef: int = 16, dt: float = 1e-4,
                 checkpoint_every: int = 50, fconv: str = "rusanov"):
        self.nr, self.nt, self.order, self.mach, self.re = nr, nt, order, mach, reynolds
        self.r1, self.stretch, self.ncoef, self.dt = r1, stretch, ncoef, dt
        self.every, self.fconv = checkpoint_every, fconv
        self.gamma = 1.4
        self.speed = mach * math.sqrt(self.gamma)  # rho = p = 1

    # -- problem set-up --
    def mesh(self, coef: Sequence[float]):
        return meshgen.cylinder_omesh(self.nr, self.nt, r0=0.5, r1=self.r1, stretch=self.stretch,
                                      wall_amp=tuple(coef))

    def params(self, alpha: float):
        V = (self.speed * math.cos(alpha), self.speed * math.sin(alpha), 0.0)
        d = {"gamma": self.gamma, "prandtl": 0.72, "mu": self.speed * 1.0 / self.re, "rt": 0.0, "c_sth": 0.0,
             "fix_vis": 1.0, "rus_k": 0.0, "ldg_b": 0.5, "ldg_tau": 0.1, "rho_fs": 1.0, "V_fs0": V[0],
             "V_fs1": V[1], "V_fs2": 0.0, "P_fs": 1.0, "T_wall": 1.0, "R_ref": 1.0, "viscous": 1.0}
        p = make_params(self.order, True, gamma=self.gamma, prandtl=0.72, mu=d["mu"], fix_vis=True,
                        ldg_b=0.5, ldg_tau=0.1, rho_fs=1.0, V_fs=V, P_fs=1.0, dt=self.dt, fconv=self.fconv)
        return p, d

    def solver(self, coef, alpha):
        mesh = self.mesh(coef)
        p, d = self.params(alpha)
        s = FRSolver(mesh, p, {"WALL": "wall_ns_adi", "FARFIELD": "char"})
        return s, mesh, d

    def initial_state(self, s, alpha):
        X = s.plan.get("coord_spts").reshape(s.nspts, 2, s.neles)
        V = (self.speed * math.cos(alpha), self.speed * math.sin(alpha))
        return ics.uniform(X, 1.0, V, 1.0, self.gamma)

    # -- objective and gradient --
    def drag(self, coef, alpha: float, nsteps: int) -> float:
        """Forward only: mean drag over nsteps RK44 steps (the library's own
        fused RK stepping and FP64 wall-force reduction)."""
        s, mesh, d = self.solver(coef, alpha)
        s.set_dt(self.dt)
        s.set_state(self.initial_state(s, alpha))
        e = np.array([math.cos(alpha), math.sin(alpha)])
        J = 0.0
        for _ in range(nsteps):
            s.step(1)
            J += float(s.wall_force()["force"][:2] @ e)
        s.close()
        return J / nsteps

    def gradient(self, coef, alpha: float, nsteps: int) -> Dict[str, object]:
        coef = np.asarray(coef, dtype=np.float64)
        s, mesh, d = self.solver(coef, alpha)
        gm = GeometryMap(s, mesh)
        wf = WallForce(s, d)
        geo0 = {k: v.detach() for k, v in gm.metrics(gm.nodes0).items()}
        c, sn = math.cos(alpha), math.sin(alpha)
        e = torch.tensor([c, sn], dtype=torch.float64, device="cuda")
        forces = []

        def objective(U, geo):
            return (wf.force(U, geo) * e).sum()

        def observe(k, U):
            # the force of each step's state (held by the solver), for the drag
            # direction's share of the angle derivative
            forces.append(s.wall_force()["force"][:2])

        traj = TrajectoryAdjoint(s, self.dt, checkpoint_every=self.every)
        U0 = self.initial_state(s, alpha)
        out = traj.run(U0, nsteps, objective, geometry=geo0, observe=observe)
        # metrics -> nodes -> wall coefficients
        X = gm.nodes0.clone().requires_grad_(True)
        m = gm.metrics(X)
        keys = list(m.keys())
        gX = torch.autograd.grad([m[k] for k in keys], X,
                                 grad_outputs=[torch.from_numpy(out["dJ_dgeometry"][k]).cuda() for k in keys])[0]
        base = np.asarray(self.mesh(np.zeros_like(coef)).nodes)[:, :2]
        dcoef = np.zeros_like(coef)
        gXn = gX.cpu().numpy()
        for k in range(len(coef)):
            ek = np.zeros_like(coef)
            ek[k] = 1.0
            phi = np.asarray(self.mesh(ek).nodes)[:, :2] - base
            dcoef[k] = float((gXn * phi).sum())
        # free-stream angle: boundary free stream, initial state, drag direction
        pbar = out["dJ_dfreestream"]
        dV = np.array([-self.speed * sn, self.speed * c])
        dalpha = float(pbar[1] * dV[0] + pbar[2] * dV[1])
        gU0 = out["dJ_dU0"]
        dU0 = torch.zeros_like(gU0)
        dU0[:, 1, :] = dV[0]  # rho = 1
        dU0[:, 2, :] = dV[1]
        dalpha += float((gU0 * dU0).sum())
        Fm = np.mean(forces, axis=0)
        dalpha += float(Fm[0] * -sn + Fm[1] * c)
        s.close()
        return {"J": out["J"], "dJ_dcoef": dcoef, "dJ_dalpha": dalpha}
