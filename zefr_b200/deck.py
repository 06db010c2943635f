"""Reader for the reference's plain-text input decks (`key value` lines and
`mesh_bound <mesh name> <bc>` lines; reference src/input.cpp:31-461), for
the keys of the residual and time-integration path.  A deck an existing
ZEFR run uses can be handed to ``FRSolver.from_deck``.

Keys that select something this library does not build (an equation other
than EulerNS, a viscous flux other than LDG, solution points other than
Legendre, implicit or pseudo-time schemes) raise ``ValueError``; keys of the
reference's I/O, restart, overset, multigrid and filter subsystems are kept
in ``Deck.raw`` and otherwise ignored.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, Optional

# deck key -> zb_deck field (zefr_b200.solver.params_from_deck)
_PARAM_KEYS = {
    "nDims": "ndims", "order": "order", "viscous": "viscous", "disable_nondim": "disable_nondim",
    "fix_vis": "fix_vis", "gamma": "gamma", "prandtl": "prandtl", "R": "R", "S": "S", "T_gas": "T_gas",
    "rho_fs": "rho_fs", "P_fs": "P_fs", "mach_fs": "mach_fs", "Re_fs": "Re_fs", "L_fs": "L_fs", "T_fs": "T_fs",
    "nx_fs": "nx_fs", "ny_fs": "ny_fs", "nz_fs": "nz_fs", "mach_wall": "mach_wall", "T_wall": "T_wall",
    "nx_wall": "nx_wall", "ny_wall": "ny_wall", "nz_wall": "nz_wall", "rus_k": "rus_k", "ldg_b": "ldg_b",
    "ldg_tau": "ldg_tau", "dt": "dt",
}
_INT_KEYS = {"nDims", "order", "viscous", "disable_nondim", "fix_vis"}
# deck keys of the explicit time schemes (FRSolver.set_time_scheme)
_TIME_KEYS = ("dt_type", "CFL", "CFL_type", "adapt_dt", "err_atol", "err_rtol", "pi_alpha", "pi_beta",
              "safety_factor", "max_factor", "min_factor", "max_dt")
_FCONV = {"rusanov": 0, "roe": 2}


@dataclass
class Deck:
    """A parsed deck: the mesh file (resolved against the deck's directory),
    the ``params_from_deck`` keywords, the boundary map, the time scheme and
    ``n_steps``; ``raw`` holds every key as written."""
    meshfile: str
    params: Dict[str, float]
    bounds: Dict[str, str]
    dt_scheme: str = "RK44"
    time_scheme: Dict[str, float] = field(default_factory=dict)
    n_steps: Optional[int] = None
    raw: Dict[str, str] = field(default_factory=dict)


def _bool(v: str) -> int:
    return int(float(v) != 0.0) if v not in ("true", "false") else int(v == "true")


def read_deck(path: str) -> Deck:
    raw: Dict[str, str] = {}
    bounds: Dict[str, str] = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if not line:
                continue
            tok = line.split()
            if tok[0] == "mesh_bound":
                if len(tok) < 3:
                    raise ValueError(f"mesh_bound needs a mesh name and a condition: {line!r}")
                if tok[1].lower() != "fluid":
                    bounds[tok[1]] = tok[2]
                continue
            raw[tok[0]] = tok[1] if len(tok) > 1 else ""
    for key in ("nDims", "meshfile", "order"):
        if key not in raw:
            raise ValueError(f"deck has no {key!r}")
    if raw.get("equation", "EulerNS") != "EulerNS":
        raise ValueError("only the EulerNS equation set is built")
    if raw.get("fvisc_type", "LDG") != "LDG":
        raise ValueError("only the LDG viscous flux is built")
    if raw.get("spt_type", "Legendre") != "Legendre":
        raise ValueError("only Legendre solution points are built")
    fconv = raw.get("fconv_type", "Rusanov").lower()
    if fconv not in _FCONV:
        raise ValueError(f"unknown fconv_type {raw['fconv_type']!r}")
    params: Dict[str, float] = {"fconv": _FCONV[fconv]}
    for key, name in _PARAM_KEYS.items():
        if key in raw:
            v = raw[key]
            params[name] = _bool(v) if key in ("viscous", "disable_nondim", "fix_vis") else (
                int(v) if key in _INT_KEYS else float(v))
    dt_scheme = raw.get("dt_scheme", "RK44")
    if dt_scheme not in ("RK44", "RK54"):
        raise ValueError(f"dt_scheme {dt_scheme!r} is not built (explicit RK44 and RK54 are)")
    ts: Dict[str, float] = {}
    for key in _TIME_KEYS:
        if key in raw:
            ts[key] = _bool(raw[key]) if key == "adapt_dt" else float(raw[key])
    mesh = raw["meshfile"]
    if not os.path.isabs(mesh):
        mesh = os.path.join(os.path.dirname(os.path.abspath(path)), mesh)
    n_steps = int(raw["n_steps"]) if "n_steps" in raw else None
    return Deck(meshfile=mesh, params=params, bounds=bounds, dt_scheme=dt_scheme, time_scheme=ts, n_steps=n_steps,
                raw=raw)
