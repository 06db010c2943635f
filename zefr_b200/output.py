"""Solution output for inspection and restart.

``write_vtu`` writes a ParaView unstructured grid in the spirit of the
reference's ``write_solution`` (src/solver.cpp:4948-5403): quadrilaterals
and hexahedra are cut into sub-cells between plot points, the solution
points plus the element boundary ([-1, x_1..x_N, 1] per direction), with the
state and the coordinates carried to the plot points by 1D Lagrange
interpolation on the solution points; triangles are written as their
solution points.  Fields: density, velocity, pressure and the conserved
variables, binary (base64) inline.

``save_state`` / ``load_state`` keep a raw FP64 copy of the state with the
time-stepping state for a resume; the reference restarts from its own .vtu
or .pyfrs files (src/solver.cpp:940-1205, 4275-4838).
"""
from __future__ import annotations

import base64
import json
import struct
from typing import Sequence

import numpy as np

VTK_VERTEX, VTK_QUAD, VTK_HEXAHEDRON = 1, 9, 12


def _lagrange(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """[len(y)][len(x)] values of the Lagrange basis on nodes x at points y."""
    L = np.ones((len(y), len(x)))
    for j, xj in enumerate(x):
        for m, xm in enumerate(x):
            if m != j:
                L[:, j] *= (y - xm) / (xj - xm)
    return L


def _apply(L: np.ndarray, A: np.ndarray, D: int, N: int) -> np.ndarray:
    """Tensor-product interpolation of A [S][C][E] (x fastest) -> [P^D][C][E]."""
    S, C, E = A.shape
    P = L.shape[0]
    if D == 2:
        a = A.reshape(N, N, C, E)                      # [y][x][C][E]
        a = np.einsum("pi,jicE->jpcE", L, a)            # x
        a = np.einsum("qj,jpcE->qpcE", L, a)            # y
        return a.reshape(P * P, C, E)
    a = A.reshape(N, N, N, C, E)                        # [z][y][x]
    a = np.einsum("pi,kjicE->kjpcE", L, a)
    a = np.einsum("qj,kjpcE->kqpcE", L, a)
    a = np.einsum("rk,kqpcE->rqpcE", L, a)
    return a.reshape(P ** 3, C, E)


def _cells(D: int, P: int, E: int) -> np.ndarray:
    """Sub-cell connectivity on a P^D plot grid per element (x fastest)."""
    loc = []
    if D == 2:
        for j in range(P - 1):
            for i in range(P - 1):
                b = i + P * j
                loc.append([b, b + 1, b + 1 + P, b + P])
    else:
        P2 = P * P
        for k in range(P - 1):
            for j in range(P - 1):
                for i in range(P - 1):
                    b = i + P * j + P2 * k
                    q = [b, b + 1, b + 1 + P, b + P]
                    loc.append(q + [v + P2 for v in q])
    loc = np.array(loc, dtype=np.int64)
    off = (np.arange(E, dtype=np.int64) * P ** D)[:, None, None]
    return (loc[None, :, :] + off).reshape(-1, loc.shape[1])


def _b64(a: np.ndarray) -> str:
    raw = np.ascontiguousarray(a).tobytes()
    return base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode("ascii")


def _da(name: str, a: np.ndarray, vtype: str, ncomp: int = 1) -> str:
    return (f'<DataArray type="{vtype}" Name="{name}" NumberOfComponents="{ncomp}" format="binary">'
            f"{_b64(a)}</DataArray>\n")


def write_vtu(path: str, solver, U: np.ndarray, gamma: float | None = None) -> None:
    """Write state U [nspts][nvars][neles] (reference layout) of ``solver`` (an
    FRSolver, or its host-only Plan)."""
    plan = getattr(solver, "plan", solver)
    info = plan.info
    D, S, V, E = info.ndims, info.nspts, info.nvars, int(info.n_eles)
    g = float(plan._params.gamma if gamma is None else gamma)
    X = plan.get("coord_spts").reshape(S, D, E)
    U = np.asarray(U, dtype=np.float64).reshape(S, V, E)
    if info.etype == 1:                                 # triangles: solution points only
        cells = np.arange(S * E, dtype=np.int64).reshape(-1, 1)
        ctype = VTK_VERTEX
        Xp = X.transpose(2, 0, 1).reshape(S * E, D)
        Up = U.transpose(2, 0, 1).reshape(S * E, V)
    else:
        N = info.order + 1
        x1 = plan.get("loc_spts").reshape(S, D)[:N, 0]
        nodes = np.concatenate([[-1.0], x1, [1.0]])
        L = _lagrange(x1, nodes)
        P = N + 2
        Xg = _apply(L, X, D, N)                          # [P^D][D][E]
        Ug = _apply(L, U, D, N)
        Xp = Xg.transpose(2, 0, 1).reshape(-1, D)
        Up = Ug.transpose(2, 0, 1).reshape(-1, V)
        cells = _cells(D, P, E)
        ctype = VTK_QUAD if D == 2 else VTK_HEXAHEDRON
    npts = Xp.shape[0]
    pts = np.zeros((npts, 3))
    pts[:, :D] = Xp
    rho = Up[:, 0]
    vel = np.zeros((npts, 3))
    vel[:, :D] = Up[:, 1:D + 1] / rho[:, None]
    p = (g - 1.0) * (Up[:, D + 1] - 0.5 * rho * (vel ** 2).sum(1))
    ncell, nv = cells.shape
    with open(path, "w") as f:
        f.write('<?xml version="1.0"?>\n')
        f.write('<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">\n')
        f.write(f'<UnstructuredGrid>\n<Piece NumberOfPoints="{npts}" NumberOfCells="{ncell}">\n')
        f.write("<Points>\n" + _da("Points", pts, "Float64", 3) + "</Points>\n")
        f.write("<Cells>\n")
        f.write(_da("connectivity", cells.reshape(-1), "Int64"))
        f.write(_da("offsets", np.arange(1, ncell + 1, dtype=np.int64) * nv, "Int64"))
        f.write(_da("types", np.full(ncell, ctype, dtype=np.uint8), "UInt8"))
        f.write("</Cells>\n<PointData>\n")
        f.write(_da("Density", rho, "Float64"))
        f.write(_da("Velocity", vel, "Float64", 3))
        f.write(_da("Pressure", p, "Float64"))
        for v in range(V):
            f.write(_da(f"U{v}", np.ascontiguousarray(Up[:, v]), "Float64"))
        f.write("</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n")


def read_vtu_array(path: str, name: str) -> np.ndarray:
    """Decode one binary DataArray of a file written by ``write_vtu``."""
    import xml.etree.ElementTree as ET
    types = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}
    for da in ET.parse(path).getroot().iter("DataArray"):
        if da.get("Name") == name:
            raw = base64.b64decode(da.text.strip())
            n = struct.unpack("<Q", raw[:8])[0]
            a = np.frombuffer(raw[8:8 + n], dtype=types[da.get("type")])
            nc = int(da.get("NumberOfComponents", "1"))
            return a.reshape(-1, nc) if nc > 1 else a
    raise KeyError(name)


def save_state(path: str, solver) -> None:
    """Raw FP64 state plus the time-stepping state (dt, error history, flow time)."""
    meta = {"nspts": solver.nspts, "nvars": solver.nvars, "neles": solver.neles, "ndims": solver.ndims,
            "order": int(solver.info.order), "time": solver.time_state()}
    np.savez(path, U=solver.get_state(), meta=json.dumps(meta))


def load_state(path: str, solver) -> dict:
    """Restore a state written by ``save_state`` into a solver of the same
    shape; returns the saved metadata (the time-stepping state is returned,
    not applied: set it with set_dt / set_time_scheme as the run needs)."""
    z = np.load(path if path.endswith(".npz") else path + ".npz", allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    shape = (solver.nspts, solver.nvars, solver.neles)
    if tuple(z["U"].shape) != shape:
        raise ValueError(f"saved state {tuple(z['U'].shape)} does not fit this solver {shape}")
    solver.set_state(z["U"])
    return meta


__all__: Sequence[str] = ("write_vtu", "read_vtu_array", "save_state", "load_state")
