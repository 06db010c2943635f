"""Long RK44 trajectories against the reference's own stepping
(FRSolver::update, src/solver.cpp:2598-2644 and step_RK 2864-3097).

The vortex workload as specified (32 x 32 quads on periodic [-5,5]^2, P3,
Rusanov, beta 5 vortex, RK44 with dt 1e-3 for 1000 steps) and a supersonic
box with inlet_sup / outlet_sup / wall_slip boundaries: the FP64 state after
each checkpoint step count against the compiled reference's.  Both runs sum
the same products in the same order except where noted in the design notes,
so the differences are rounding that grows with the step count; the bound is
1e-12 relative per variable at every checkpoint.
"""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200.solver import FRSolver, params_from_reference

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", gc.traj_names())
def test_trajectory_matches_reference(name):
    t = gc.load_traj(name)
    s = FRSolver(t.mesh, params_from_reference(t.params, t.order), t.bounds)
    s.set_state(t.U0)
    done, errs = 0, []
    for k, ref in zip(t.meta["checkpoints"], t.states):
        s.step(k - done)
        done = k
        errs.append(gc.rel_err(s.get_state(), ref))
    print(name, dict(zip(t.meta["checkpoints"], errs)))
    assert max(errs) < 1e-12, errs
