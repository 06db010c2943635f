"""The allocation-free residual entry point, called through the C ABI.

zb_compute_residual_noalloc exists for callers that cannot call cudaMalloc
when they need a residual (an application that owns all device memory through
its own allocator, a sandboxed plugin, a loop that must stay out of the
driver's allocator): they pass device state and residual buffers they already
own, and the library keeps every intermediate in one static device array.
This test owns its buffers through torch, calls the entry point twice in a row
on each mesh, and compares with the allocating zb_compute_residual path.  It
sits in its own file so a run stopping at the first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

import golden_cases as gc
from zefr_b200 import _lib, meshgen
from zefr_b200.solver import FRSolver, Plan, make_params, params_from_reference

pytestmark = pytest.mark.gpu

_DP = ctypes.POINTER(ctypes.c_double)


def _noalloc(plan, U_dev, out_dev, stream=None):
    return _lib.lib().zb_compute_residual_noalloc(plan.h, ctypes.cast(U_dev.data_ptr(), _DP),
                                                  ctypes.cast(out_dev.data_ptr(), _DP), stream)


@pytest.mark.parametrize("name", ["quad_p3_euler_vortex", "hex_p3_ns_tgv", "hex_p1_ns", "hex_p2_euler_jitter",
                                  "hex_p4_euler", "cyl_p3_ns_char_adi"])
def test_noalloc_matches_allocating_path(name):
    import torch
    g = gc.load(name)
    params = params_from_reference(g.params, g.order)
    ref = FRSolver(g.mesh, params, g.bounds).residual(g.U0, 0)
    plan = Plan(g.mesh, params, g.bounds)
    U = torch.from_numpy(g.U0).cuda()
    for _ in range(2):  # second call reuses the shared array left by the first
        out = torch.full_like(U, float("nan"))
        st = _noalloc(plan, U, out)
        assert st == 0, _lib.lib().zb_last_error().decode()
        torch.cuda.synchronize()
        R = out.cpu().numpy()
        # same FP64 kernels as the allocating path: 1e-12 relative per variable
        assert gc.rel_err(R, ref) < 1e-12
        assert gc.rel_err(R, g.R0) < 1e-12


def test_noalloc_rejects_meshes_beyond_its_array():
    import torch
    plan = Plan(meshgen.box_hexes(16, 16, 16), make_params(3, True, mu=1e-3), {"PERIODIC": "periodic"})
    n = plan.info.nspts * plan.info.nvars * plan.info.n_eles
    U = torch.zeros(n, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(U)
    st = _noalloc(plan, U, out)
    assert st == -1  # ZB_ERR_ARG
    msg = _lib.lib().zb_last_error().decode()
    assert "scratch" in msg and "33554432" in msg
