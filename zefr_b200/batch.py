"""Batched RK stepping of many independent Euler cases (``zb_batch_*``).

``vortex_cases`` builds the batched-vortex workload: independent periodic
quad meshes n x n on [-5,5]^2, order P, each carrying an isentropic vortex of
strength beta at a seeded centre on a uniform stream of Mach Ma, all drawn
from one seed.  ``Batch`` advances them together: one persistent launch per
RK stage for all cases, the four stages of a step captured as a CUDA graph,
launch shape chosen by ``autotune``.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib, ics, meshgen
from ._lib import check, lib
from .solver import FRSolver, make_params


def vortex_case_params(ncases: int, seed: int, n_range=(8, 96), orders=(1, 5), dt_cfl: float = 0.1,
                       gamma: float = 1.4) -> List[dict]:
    """Parameters of the seeded batched-vortex workload, one dict per case:
    mesh size n (n x n quads on [-5,5]^2) and order P uniform in their
    ranges, vortex centre uniform in [-2,2]^2, strength beta uniform in
    [1,5], stream Mach uniform in [0.2,0.8], and dt = dt_cfl * h /
    ((Ma + 1) c (P + 1)^2) (a fixed fraction of the explicit stability
    limit)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(ncases):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        P = int(rng.integers(orders[0], orders[1] + 1))
        center = rng.uniform(-2.0, 2.0, size=2)
        beta = float(rng.uniform(1.0, 5.0))
        mach = float(rng.uniform(0.2, 0.8))
        c = math.sqrt(gamma)
        h = 10.0 / n
        dt = dt_cfl * h / ((mach + 1.0) * c * (P + 1) ** 2)
        out.append({"n": n, "P": P, "center": center.tolist(), "beta": beta, "mach": mach, "dt": dt})
    return out


def vortex_cases(ncases: int, seed: int, n_range=(8, 96), orders=(1, 5), precision: str = "mixed",
                 dt_cfl: float = 0.1) -> List[FRSolver]:
    """Seeded batched-vortex workload (vortex_case_params): one solver per
    case with the vortex state set; the parameters are kept as ``s.case``."""
    gamma = 1.4
    c = math.sqrt(gamma)
    out = []
    for case in vortex_case_params(ncases, seed, n_range, orders, dt_cfl, gamma):
        n, P = case["n"], case["P"]
        p = make_params(P, False, gamma=gamma, precision=precision, dt=case["dt"])
        s = FRSolver(meshgen.box_quads(n, n), p, {"PERIODIC": "periodic"})
        X = s.plan.get("coord_spts").reshape(s.nspts, 2, s.neles)
        s.set_state(ics.isentropic_vortex(X, beta=case["beta"], center=tuple(case["center"]),
                                          u_inf=(case["mach"] * c, 0.0), gamma=gamma))
        s.case = case
        out.append(s)
    return out


class Batch:
    """Many FRSolver contexts stepped as one batch (Euler, quadrilaterals)."""

    def __init__(self, solvers: Sequence[FRSolver]):
        self.solvers = list(solvers)
        arr = (ctypes.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        h = ctypes.c_void_p()
        check(lib().zb_batch_create(arr, len(self.solvers), ctypes.byref(h)))
        self.h = h

    @property
    def dof(self) -> int:
        return sum(s.nspts * s.nvars * s.neles for s in self.solvers)

    def step(self, n: int = 1, graph: bool = True) -> None:
        check(lib().zb_batch_step(self.h, n, 1 if graph else 0))

    def stage(self, stage: int) -> None:
        check(lib().zb_batch_stage(self.h, stage))

    def synchronize(self) -> None:
        check(lib().zb_batch_synchronize(self.h))

    def autotune(self, steps: int = 3, form: Optional[bool] = None) -> Dict[str, float]:
        """Time every launch shape and install the fastest; form True keeps
        to one kernel per stage for all orders, False to one kernel per order,
        None takes either."""
        c = _lib.ZbBatchConfig()
        check(lib().zb_batch_autotune_form(self.h, steps, -1 if form is None else int(bool(form)), ctypes.byref(c)))
        return {"threads": c.threads, "group": c.group, "chunk": c.chunk, "blocks_per_sm": c.blocks_per_sm,
                "order": c.order, "ms_per_step": c.ms_per_step, "fused": c.fused}

    def set_config(self, threads: int, blocks_per_sm: int, order: int = 0, group: int = 64, chunk: int = 1,
                   fused: bool = False) -> None:
        c = _lib.ZbBatchConfig(threads, blocks_per_sm, order, 0.0, group, chunk, int(bool(fused)))
        check(lib().zb_batch_set_config(self.h, ctypes.byref(c)))

    def launch_count(self) -> int:
        return int(lib().zb_batch_launch_count(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().zb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
