"""PyTorch autograd over the DFR residual and RK44 trajectories.

``residual(U, solver)`` is a differentiable residual: its backward calls the
library's hand-written adjoint (``zb_vjp``), never a PyTorch trace of the
kernels.  ``TrajectoryAdjoint`` differentiates a time-averaged objective over
RK44 steps (``FRSolver::step_RK`` with the RK44 tables of src/solver.cpp:
722-735) with respect to the initial state and the free-stream state, storing
a checkpoint every ``checkpoint_every`` steps and recomputing the states of
each segment during the reverse sweep; each step's transpose is one library
call (``zb_rk_step_vjp``) that re-runs the four stages and applies their
adjoints on the device.

Everything is plain FP64 on the device: the adjoint exists for ZB_FP64
contexts only.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Optional, Tuple

import numpy as np
import torch

from .solver import FRSolver


class _Residual(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U: torch.Tensor, solver: FRSolver, stage: int):
        solver.set_state(U)
        solver.compute_residual(stage)
        R = torch.empty_like(U)
        solver.get_residual_device(R, stage)
        ctx.solver = solver
        ctx.save_for_backward(U)
        return R

    @staticmethod
    def backward(ctx, gR: torch.Tensor):
        (U,) = ctx.saved_tensors
        ctx.solver.set_state(U)
        return ctx.solver.vjp(gR.contiguous()), None, None


def residual(U: torch.Tensor, solver: FRSolver, stage: int = 0) -> torch.Tensor:
    """divF(U) in the reference layout [spt][var][ele] (float64 CUDA tensor),
    differentiable with respect to U through the library's adjoint."""
    if U.dtype != torch.float64 or not U.is_cuda:
        raise TypeError("residual() takes a float64 CUDA tensor")
    return _Residual.apply(U.contiguous(), solver, stage)


def _device_array(solver: FRSolver, name: str, shape) -> torch.Tensor:
    return torch.from_numpy(solver.plan.get(name).reshape(shape)).cuda()


class TrajectoryAdjoint:
    """Gradient of J = (1/n) sum_{k=1..n} j(U_k) over n RK44 steps.

    ``objective(U) -> scalar tensor`` is any differentiable torch function of
    the state (e.g. :func:`kinetic_energy`); its state gradient comes from
    torch autograd, the residual's from the library adjoint.  The free-stream
    gradient covers rho_fs, V_fs[0..2], P_fs.
    """

    def __init__(self, solver: FRSolver, dt: float, checkpoint_every: int = 50):
        self.s = solver
        self.dt = float(dt)
        self.every = int(checkpoint_every)
        solver.set_dt(self.dt)

    # -- forward pieces --
    def _step(self, U: torch.Tensor) -> torch.Tensor:
        """One RK44 step by the library's fused stages (the stepping the
        forward objective runs use), back as a torch tensor."""
        self.s.set_state(U)
        self.s.step(1)
        out = torch.empty_like(U)
        self.s.get_state_device(out)
        return out

    # -- reverse pieces --
    def _step_adjoint(self, U0: torch.Tensor, Ubar_new: torch.Tensor, pbar: np.ndarray, gbar=None) -> torch.Tensor:
        """(dU1/dU0)^T Ubar_new for the RK44 step from U0: one library call
        (zb_rk_step_vjp) that recomputes the four stages and applies the four
        stage adjoints with the RK weights on the device; with ``gbar`` the
        metric adjoint (residuals and the update's 1/|J|) goes to the
        library's device-side sums."""
        return self.s.rk_step_vjp(U0, Ubar_new, pbar, geometry=gbar is not None)

    @staticmethod
    def _obj_grad_batch(objective: Callable, Us: torch.Tensor, geo=None):
        """Objective values and gradients for a stack of states Us [M,S,V,E]
        in one vectorised evaluation (torch.func.vmap of grad_and_value): the
        sum of the values, the state gradients per state and, with ``geo``,
        the geometry gradient summed over the stack.  Falls back to one
        autograd call per state when the objective cannot be vectorised."""
        try:
            from torch.func import grad_and_value, vmap
            if geo is None:
                gU, j = vmap(grad_and_value(objective))(Us)
                return float(j.sum()), gU, None
            leaves = {k: v.detach() for k, v in geo.items()}
            (gU, gG), j = vmap(grad_and_value(objective, argnums=(0, 1)), in_dims=(0, None))(Us, leaves)
            return float(j.sum()), gU, {k: v.sum(dim=0) for k, v in gG.items()}
        except Exception:  # noqa: BLE001 -- objective not vmap-able: per-state autograd
            gUs, gsum, jsum = [], None, 0.0
            for U in Us:
                j, gU, gG = TrajectoryAdjoint._obj_grad(objective, U, geo)
                jsum += j
                gUs.append(gU)
                if gG is not None:
                    gsum = gG if gsum is None else {k: gsum[k] + gG[k] for k in gsum}
            return jsum, torch.stack(gUs), gsum

    @staticmethod
    def _obj_grad(objective: Callable, U: torch.Tensor, geo=None):
        x = U.detach().clone().requires_grad_(True)
        if geo is None:
            j = objective(x)
            (g,) = torch.autograd.grad(j, x)
            return float(j.detach()), g, None
        leaves = {k: v.detach().clone().requires_grad_(True) for k, v in geo.items()}
        j = objective(x, leaves)
        grads = torch.autograd.grad(j, [x] + list(leaves.values()))
        return float(j.detach()), grads[0], dict(zip(leaves, grads[1:]))

    def run(self, U0, nsteps: int, objective: Callable, geometry=None,
            observe: Optional[Callable] = None) -> Dict[str, object]:
        """Returns J, dJ/dU0 (CUDA tensor) and dJ/d(rho_fs, V_fs[0..2], P_fs).

        With ``geometry`` (a dict of the current metric tensors, as
        ``geometry.GeometryMap.metrics`` returns them), ``objective(U, geo)``
        also takes the metrics and the result adds ``dJ_dgeometry``: the
        gradient with respect to inv_jaco, jaco_det, norm and dA, summed over
        the residual's adjoint, the RK update's 1/|J| and the objective.

        The forward sweep only steps (the library's fused RK44) and keeps
        checkpoints; the objective is evaluated, with its gradients, on the
        states the reverse sweep recomputes, a segment at a time.
        ``observe(k, U)``, if given, sees every forward state U_k while the
        solver holds it."""
        U = torch.as_tensor(U0, dtype=torch.float64).cuda().contiguous()
        checkpoints = {0: U.clone()}
        obj_grad_fn = objective
        J = 0.0
        with torch.no_grad():
            for k in range(1, nsteps + 1):
                U = self._step(U)
                if observe is not None:
                    observe(k, U)
                if k % self.every == 0:
                    checkpoints[k] = U.clone()
        # reverse sweep, one checkpointed segment at a time from the end
        Ubar = torch.zeros_like(U)
        pbar = np.zeros(5)
        gbar = None
        if geometry is not None:
            # the objective's and the RK update's parts, on the device
            gbar = {k: torch.zeros_like(v) for k, v in geometry.items()}
        starts = [k for k in sorted(checkpoints) if k < nsteps]
        for i in range(len(starts) - 1, -1, -1):
            k0 = starts[i]
            k1 = starts[i + 1] if i + 1 < len(starts) else nsteps
            # states[m] = U_{k0+m}, recomputed from the checkpoint
            states = [checkpoints[k0]]
            for _ in range(k0 + 1, k1):
                states.append(self._step(states[-1]))
            last = checkpoints[k1] if k1 in checkpoints else self._step(states[-1])
            # the objective's gradients at U_{k0+1..k1} do not depend on the
            # adjoint: vectorised evaluations over the segment, in chunks of
            # about 1 GiB of states
            nexts = states[1:] + [last]
            chunk = max(1, (1 << 30) // max(1, last.numel() * last.element_size()))
            gUs = []
            for c0 in range(0, len(nexts), chunk):
                jsum, gU, gGsum = self._obj_grad_batch(obj_grad_fn, torch.stack(nexts[c0:c0 + chunk]), geometry)
                J += jsum / nsteps
                gUs.extend(gU.unbind(0))
                if gGsum is not None:
                    for k in gbar:
                        gbar[k] += gGsum[k] / nsteps
            for m in range(k1 - k0 - 1, -1, -1):
                Ubar = Ubar + gUs[m] / nsteps
                Ubar = self._step_adjoint(states[m], Ubar, pbar, gbar)
        out = {"J": J, "dJ_dU0": Ubar, "dJ_dfreestream": pbar}
        if gbar is not None:
            lib_part = self.s.geometry_adjoint(reset=True)
            out["dJ_dgeometry"] = {k: gbar[k].cpu().numpy() + lib_part[k] for k in gbar}
        return out


def kinetic_energy(solver: FRSolver) -> Callable[[torch.Tensor], torch.Tensor]:
    """Volume integral of 1/2 rho |u|^2 (report_turbulent_stats,
    src/solver.cpp:7813-7917) as a torch function of the state."""
    S, V, E = solver.state_shape
    jw = (_device_array(solver, "jaco_det_spts", (S, E)) *
          torch.from_numpy(solver.plan.get("weights_spts")).cuda().reshape(S, 1))

    def f(U: torch.Tensor) -> torch.Tensor:
        rho = U[:, 0, :]
        m2 = (U[:, 1:V - 1, :] ** 2).sum(dim=1)
        return (jw * 0.5 * m2 / rho).sum()

    return f
