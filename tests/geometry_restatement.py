"""Torch restatement of the set-up metrics as functions of the mesh node
coordinates (reference src/elements.cpp:325-407, 845-996): the checker of the
library's geometry kernels (zb_geometry_eval and its adjoint) and the CPU
source of metrics for the wall-force restatement test.  Test infrastructure
only."""
from typing import Dict, Tuple

import numpy as np
import torch


def _t(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


def _adjugate(J: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """J [Dref, P, Dphys, E] -> (adjugate in the reference inv_jaco layout
    [D, P, D, E], determinant [P, E]); 2D and 3D as the set-up computes them."""
    D = J.shape[0]
    if D == 2:
        det = J[0, :, 0] * J[1, :, 1] - J[0, :, 1] * J[1, :, 0]
        inv = torch.stack([torch.stack([J[1, :, 1], -J[1, :, 0]], dim=1),
                           torch.stack([-J[0, :, 1], J[0, :, 0]], dim=1)], dim=0)
        return inv, det
    xr, xs, xt = J[0, :, 0], J[1, :, 0], J[2, :, 0]
    yr, ys, yt = J[0, :, 1], J[1, :, 1], J[2, :, 1]
    zr, zs, zt = J[0, :, 2], J[1, :, 2], J[2, :, 2]
    det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr)
    rows = [[ys * zt - yt * zs, xt * zs - xs * zt, xs * yt - xt * ys],
            [yt * zr - yr * zt, xr * zt - xt * zr, xt * yr - xr * yt],
            [yr * zs - ys * zr, xs * zr - xr * zs, xr * ys - xs * yr]]
    inv = torch.stack([torch.stack(r, dim=1) for r in rows], dim=0)
    return inv, det


class GeometryRestatement:
    """Set-up metrics of a solver's plan as torch functions of node coordinates."""

    def __init__(self, solver, mesh, device="cuda"):
        p = solver.plan
        D, S, E, Fp = solver.ndims, solver.nspts, solver.neles, solver.info.nfpts
        nn = mesh.elements.shape[1]
        self.D, self.S, self.E, self.Fp = D, S, E, Fp
        self.dev = device
        self.dss = _t(p.get("dshape_spts").reshape(D, S, nn), device)
        self.dsf = _t(p.get("dshape_fpts").reshape(D, Fp, nn), device)
        self.tn = _t(p.get("tnorm").reshape(Fp, D), device)
        self.e2n = torch.as_tensor(np.asarray(mesh.elements, dtype=np.int64), device=device)
        part = p.get("fpt_partner").reshape(Fp, E).astype(np.int64)
        slot = p.get("fpt_slot").reshape(Fp, E).astype(np.int64)
        right = (part >= 0) & (slot == 1)
        self.right = torch.as_tensor(right, device=device)
        self.pe = torch.as_tensor(np.where(right, part // Fp, 0), device=device)
        self.pf = torch.as_tensor(np.where(right, part % Fp, 0), device=device)
        self.nodes0 = _t(np.asarray(mesh.nodes)[:, :D], device)

    def metrics(self, X: torch.Tensor) -> Dict[str, torch.Tensor]:
        """X [n_nodes, D] -> inv_jaco [D,S,D,E], jaco_det [S,E], norm [Fp,D,E], dA [Fp,E]."""
        nodes = X[self.e2n]                                   # [E, nn, D]
        Js = torch.einsum("asn,end->asde", self.dss, nodes)
        inv, det = _adjugate(Js)
        Jf = torch.einsum("afn,end->afde", self.dsf, nodes)
        invf, _ = _adjugate(Jf)                               # [D, Fp, D, E]
        norm = torch.einsum("bfae,fb->fae", invf, self.tn)    # sum_d2 inv[d2][f][d1] tnorm[f][d2]
        dA = torch.sqrt((norm * norm).sum(dim=1))
        n_own = norm / dA[:, None, :]
        n_left = n_own[self.pf, :, self.pe]                   # [Fp, E, D]
        fnorm = torch.where(self.right[:, None, :], n_left.permute(0, 2, 1), n_own)
        return {"inv_jaco": inv, "jaco_det": det, "norm": fnorm, "dA": dA}
