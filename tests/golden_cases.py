"""Loading helpers for the golden fixtures written by tests/golden/make_golden.py."""
from __future__ import annotations

import glob
import json
import os
from dataclasses import dataclass
from typing import Dict, List

import numpy as np

from oracle.dfr_numpy import Setup
from zefr_b200.meshgen import Mesh

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@dataclass
class Golden:
    name: str
    meta: Dict
    mesh: Mesh
    bounds: Dict[str, str]
    params: Dict[str, float]
    U0: np.ndarray
    R0: np.ndarray
    Un: np.ndarray
    setup_arrays: Dict[str, np.ndarray]

    @property
    def viscous(self) -> bool:
        return bool(self.meta["viscous"])

    @property
    def order(self) -> int:
        return int(self.meta["order"])

    def setup(self) -> Setup:
        S, V, E = self.meta["shape"]
        return Setup.from_arrays(self.meta["ndims"], S, self.meta["nfpts"], E, lambda k: self.setup_arrays[k])


def names() -> List[str]:
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz")))


def load(name: str) -> Golden:
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"), allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    faces = []
    for t, nodes, nm in zip(z["faces_type"], z["faces_nodes"], z["faces_name"]):
        faces.append((int(t), tuple(int(n) for n in nodes if n >= 0), str(nm)))
    mesh = Mesh(ndims=meta["ndims"], nodes=z["nodes"], gmsh_type=meta["gmsh_type"], elements=z["elements"],
                bnd_faces=faces)
    setup = {k[len("setup_"):]: z[k] for k in z.files if k.startswith("setup_")}
    return Golden(name=name, meta=meta, mesh=mesh, bounds=meta["bounds"], params=meta["params"], U0=z["U0"],
                  R0=z["R0"], Un=z["Un"], setup_arrays=setup)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a-b| over the tensor, relative to the largest |b| of the same variable."""
    scale = np.abs(b).max(axis=(0, 2), keepdims=True)
    return float((np.abs(a - b) / np.maximum(scale, 1e-300)).max())


TIME_DIR = os.path.join(GOLDEN_DIR, "time")


@dataclass
class TimeGolden:
    """Time-integration fixture: mesh, deck, U0, the reference's dt(0) after
    every step (dt0), its per-element dt after the last step (dt_ele) and the
    final state (Un)."""
    name: str
    meta: Dict
    mesh: Mesh
    bounds: Dict[str, str]
    params: Dict[str, float]
    U0: np.ndarray
    Un: np.ndarray
    dt0: np.ndarray
    dt_ele: np.ndarray

    @property
    def viscous(self) -> bool:
        return bool(self.meta["viscous"])

    @property
    def order(self) -> int:
        return int(self.meta["order"])

    @property
    def deck(self) -> Dict:
        return self.meta["deck"]


def time_names() -> List[str]:
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(TIME_DIR, "*.npz")))


def load_time(name: str) -> TimeGolden:
    z = np.load(os.path.join(TIME_DIR, name + ".npz"), allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    faces = []
    for t, nodes, nm in zip(z["faces_type"], z["faces_nodes"], z["faces_name"]):
        faces.append((int(t), tuple(int(n) for n in nodes if n >= 0), str(nm)))
    mesh = Mesh(ndims=meta["ndims"], nodes=z["nodes"], gmsh_type=meta["gmsh_type"], elements=z["elements"],
                bnd_faces=faces)
    return TimeGolden(name=name, meta=meta, mesh=mesh, bounds=meta["bounds"], params=meta["params"], U0=z["U0"],
                      Un=z["Un"], dt0=z["dt0"], dt_ele=z["dt_ele"])


DIAG_DIR = os.path.join(GOLDEN_DIR, "diag")


def diag_names() -> List[str]:
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(DIAG_DIR, "*.npz")))


def load_diag(name: str) -> Dict[str, np.ndarray]:
    """The reference's own diagnostics at the golden case's U0 after
    compute_residual(0): res_max / res_l1 / res_l2 (report_residuals, per
    variable, divided by the solution point count), turb = (ke, enstrophy,
    normaliser) of report_turbulent_stats (3D Navier-Stokes cases), force and
    moment of compute_moments (cases with walls)."""
    z = np.load(os.path.join(DIAG_DIR, name + ".npz"), allow_pickle=False)
    return {k: z[k] for k in z.files}


TRAJ_DIR = os.path.join(GOLDEN_DIR, "traj")


@dataclass
class TrajGolden:
    """Long RK44 trajectory of the reference: U0 and the state after each
    step count in meta["checkpoints"] (states[i])."""
    name: str
    meta: Dict
    mesh: Mesh
    bounds: Dict[str, str]
    params: Dict[str, float]
    U0: np.ndarray
    states: np.ndarray

    @property
    def viscous(self) -> bool:
        return bool(self.meta["viscous"])

    @property
    def order(self) -> int:
        return int(self.meta["order"])


def traj_names() -> List[str]:
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(TRAJ_DIR, "*.npz")))


def load_traj(name: str) -> TrajGolden:
    z = np.load(os.path.join(TRAJ_DIR, name + ".npz"), allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    faces = []
    for t, nodes, nm in zip(z["faces_type"], z["faces_nodes"], z["faces_name"]):
        faces.append((int(t), tuple(int(n) for n in nodes if n >= 0), str(nm)))
    mesh = Mesh(ndims=meta["ndims"], nodes=z["nodes"], gmsh_type=meta["gmsh_type"], elements=z["elements"],
                bnd_faces=faces)
    return TrajGolden(name=name, meta=meta, mesh=mesh, bounds=meta["bounds"], params=meta["params"], U0=z["U0"],
                      states=z["states"])


def comp_err(a: np.ndarray, b: np.ndarray, floor: float = 1e-2) -> float:
    """Largest relative difference per component, |a-b| / |b|, over the
    components whose magnitude is at least ``floor`` times the largest |b| of
    the same variable (below that, a component is a cancellation residue
    whose relative difference measures nothing)."""
    scale = np.abs(b).max(axis=(0, 2), keepdims=True)
    mask = np.abs(b) >= floor * scale
    return float((np.abs(a - b)[mask] / np.abs(b)[mask]).max())
