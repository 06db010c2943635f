"""Triangle Navier-Stokes residual of the mixed form with the gradient
kernel's operator products on the tensor pipe (zb_params.tensor_ops = 1:
tcgen05 MMAs, TF32x3 split products, FP32 accumulation) against the
reference's golden residuals, the CUDA-core mixed kernel and the FP64 form.

The products are the reference's oppD U + oppD_fpts Ucomm, oppE dU and
oppDiv F (src/elements.cpp:1362-1474); TF32x3 keeps about 21 bits of each
operand, so the tensor-core form stays within the mixed form's own bound
against the reference (1e-5 relative L2 on the golden cases)."""
import numpy as np
import pytest

import golden_cases as gc
from zefr_b200 import ics, meshgen
from zefr_b200.solver import FRSolver, make_params, params_from_reference

pytestmark = pytest.mark.gpu

TRI_NS = ["tri_p4_ns_jitter", "tri_p1_ns_adi"]


def _solver(g, **kw):
    return FRSolver(g.mesh, params_from_reference(g.params, g.order, precision="mixed", **kw), g.bounds)


@pytest.mark.parametrize("name", TRI_NS)
def test_tensor_core_residual_matches_reference(name):
    g = gc.load(name)
    R = _solver(g, tensor_ops=True).residual(g.U0, 0)
    Rc = _solver(g).residual(g.U0, 0)
    nrm = np.linalg.norm(g.R0)
    assert np.linalg.norm(R - g.R0) / nrm < 1e-5
    # and with the CUDA-core products: the same FP32 arithmetic up to the
    # order of the sums and the split products' rounding
    assert np.linalg.norm(R - Rc) / nrm < 1e-5


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_tensor_core_residual_every_order(order):
    """P1-P4 (K and N of the products padded to the MMA shapes), a mesh whose
    tile count is not a multiple of the four tiles a CTA takes, periodic, Roe,
    against the FP64 form."""
    mesh = meshgen.box_tris(7, seed=order, jitter=0.15)  # 98 triangles: 13 tiles
    common = dict(mu=2e-3, prandtl=0.71, ldg_b=0.5, ldg_tau=0.1, fconv="roe", V_fs=(0.2, 0.0, 0.0))
    out = {}
    for key, kw in (("fp64", dict(precision="fp64")), ("mixed", dict(precision="mixed")),
                    ("tc", dict(precision="mixed", tensor_ops=True))):
        s = FRSolver(mesh, make_params(order, True, **common, **kw), {"PERIODIC": "periodic"})
        X = s.plan.get("coord_spts").reshape(s.nspts, 2, s.neles)
        U = ics.double_shear_layer(X, mach=0.2, noise=1e-2, seed=order)
        out[key] = s.residual(U, 1)
    nrm = np.linalg.norm(out["fp64"])
    e_tc = np.linalg.norm(out["tc"] - out["fp64"]) / nrm
    e_cc = np.linalg.norm(out["mixed"] - out["fp64"]) / nrm
    assert e_tc < 1e-4
    assert e_tc < 4 * e_cc + 1e-6


def test_tensor_core_steps_and_functionals():
    """RK44 steps (the face kernel's RK update after the tensor-core gradient
    kernel) and the enstrophy functional (the kernel's gradient output) track
    the CUDA-core mixed form."""
    g = gc.load("tri_p4_ns_jitter")
    a, b = _solver(g, tensor_ops=True), _solver(g)
    for s in (a, b):
        s.set_state(g.U0)
        s.step(5)
    Ua, Ub = a.get_state(), b.get_state()
    assert np.linalg.norm(Ua - Ub) / np.linalg.norm(Ub) < 1e-6
    fa, fb = a.functionals(), b.functionals()
    assert abs(fa["enstrophy"] - fb["enstrophy"]) <= 1e-5 * abs(fb["enstrophy"])
    assert abs(fa["ke"] - fb["ke"]) <= 1e-6 * abs(fb["ke"])


def test_tensor_ops_rejected_outside_triangle_mixed_ns():
    from zefr_b200._lib import ZbError
    with pytest.raises(ZbError) as ei:
        FRSolver(meshgen.box_quads(4, 4), make_params(2, True, mu=1e-3, tensor_ops=True, precision="mixed"),
                 {"PERIODIC": "periodic"})
    assert "tensor" in str(ei.value)
