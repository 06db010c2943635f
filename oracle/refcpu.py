"""ctypes driver for the reference's own CPU solver (test infrastructure only).

Loads ``oracle/_ref/libzefr_ref.so`` (parity build) or
``oracle/_ref/libzefr_ref_fast.so`` (release-flag build used for CPU timing),
both compiled by ``oracle/Makefile`` from the reference sources, and drives
``FRSolver`` through ``oracle/ref_harness.cpp``.  Only tests, the golden-fixture
script, ``smoke()`` and the benchmark's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PARITY = os.path.join(HERE, "_ref", "libzefr_ref.so")
LIB_FAST = os.path.join(HERE, "_ref", "libzefr_ref_fast.so")

PARAM_NAMES = ["gamma", "prandtl", "mu", "rt", "c_sth", "fix_vis", "rus_k", "ldg_b", "ldg_tau",
               "rho_fs", "V_fs0", "V_fs1", "V_fs2", "P_fs", "T_wall", "R_ref", "V_wall0", "V_wall1",
               "V_wall2", "dt", "viscous", "T_tot_fs", "P_tot_fs"]

_libs: Dict[str, ctypes.CDLL] = {}


def available(fast: bool = False) -> bool:
    return os.path.exists(LIB_FAST if fast else LIB_PARITY)


def _lib(fast: bool) -> ctypes.CDLL:
    path = LIB_FAST if fast else LIB_PARITY
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle`")
        lib = ctypes.CDLL(path)
        lib.zr_create.restype = ctypes.c_void_p
        lib.zr_create.argtypes = [ctypes.c_char_p]
        lib.zr_destroy.argtypes = [ctypes.c_void_p]
        lib.zr_last_error.restype = ctypes.c_char_p
        for fn in ("zr_info",):
            getattr(lib, fn).argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]
        lib.zr_params.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.zr_set_state.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.zr_get_state.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.zr_compute_residual.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.zr_get_residual.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        lib.zr_update.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.zr_report_residuals.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        lib.zr_turbulent_stats.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
        lib.zr_compute_moments.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.zr_get_array.restype = ctypes.c_long
        lib.zr_get_array.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), ctypes.c_long]
        _libs[path] = lib
    return _libs[path]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class RefSolver:
    """One reference ``FRSolver`` built from a deck file."""

    def __init__(self, deck: str, fast: bool = False):
        self.lib = _lib(fast)
        cwd = os.getcwd()
        # the reference creates its output directory relative to the cwd
        os.chdir(os.path.dirname(os.path.abspath(deck)))
        try:
            h = self.lib.zr_create(os.path.basename(deck).encode())
        finally:
            os.chdir(cwd)
        if not h:
            raise RuntimeError("reference setup failed: " + self.lib.zr_last_error().decode())
        self.h = ctypes.c_void_p(h)
        info = (ctypes.c_int * 12)()
        self.lib.zr_info(self.h, info)
        (self.ndims, self.nvars, self.nspts, self.nfpts, self.neles, self.nelespad, self.nstages,
         self.ngfpts, self.ngfpts_int, self.ngfpts_bnd, self.etype_id, self.order) = list(info)
        p = np.zeros(23)
        self.lib.zr_params(self.h, _dp(p))
        self.params = dict(zip(PARAM_NAMES, p.tolist()))

    def close(self) -> None:
        if self.h:
            self.lib.zr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def state_shape(self):
        return (self.nspts, self.nvars, self.neles)

    def set_state(self, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == self.state_shape
        self.lib.zr_set_state(self.h, _dp(U))

    def get_state(self) -> np.ndarray:
        U = np.empty(self.state_shape)
        self.lib.zr_get_state(self.h, _dp(U))
        return U

    def compute_residual(self, stage: int = 0) -> None:
        if self.lib.zr_compute_residual(self.h, stage) != 0:
            raise RuntimeError(self.lib.zr_last_error().decode())

    def get_residual(self, stage: int = 0) -> np.ndarray:
        out = np.empty(self.state_shape)
        self.lib.zr_get_residual(self.h, stage, _dp(out))
        return out

    def residual(self, U: np.ndarray, stage: int = 0) -> np.ndarray:
        self.set_state(U)
        self.compute_residual(stage)
        return self.get_residual(stage)

    def update(self, nsteps: int = 1) -> None:
        if self.lib.zr_update(self.h, nsteps) != 0:
            raise RuntimeError(self.lib.zr_last_error().decode())

    def report_residuals(self, res_type: int) -> np.ndarray:
        """The per-variable residual the reference's report_residuals prints
        for ``res_type`` (0 max, 1 L1, 2 L2 of divF/|J|, divided by the number
        of solution points) after the last compute_residual."""
        out = np.zeros(self.nvars)
        if self.lib.zr_report_residuals(self.h, res_type, _dp(out)) != 0:
            raise RuntimeError(self.lib.zr_last_error().decode())
        return out

    def turbulent_stats(self) -> Dict[str, float]:
        """Kinetic energy and enstrophy as the reference's
        report_turbulent_stats writes them (normalised by vol rho_fs |V_fs|^2),
        with that normaliser, after the last compute_residual."""
        import tempfile
        out = np.zeros(3)
        with tempfile.TemporaryDirectory() as tmp:
            path = os.path.join(tmp, "turb_stats.dat")
            if self.lib.zr_turbulent_stats(self.h, path.encode(), _dp(out)) != 0:
                raise RuntimeError(self.lib.zr_last_error().decode())
        return {"ke": float(out[0]), "enstrophy": float(out[1]), "norm": float(out[2])}

    def compute_moments(self) -> Dict[str, np.ndarray]:
        """Wall force and moment of the reference's compute_moments after the
        last compute_residual."""
        out = np.zeros(6)
        if self.lib.zr_compute_moments(self.h, _dp(out)) != 0:
            raise RuntimeError(self.lib.zr_last_error().decode())
        return {"force": out[:3].copy(), "moment": out[3:].copy()}

    def array(self, name: str) -> np.ndarray:
        n = self.lib.zr_get_array(self.h, name.encode(), None, 0)
        if n < 0:
            raise KeyError(name)
        out = np.empty(n)
        self.lib.zr_get_array(self.h, name.encode(), _dp(out), n)
        return out


def write_deck(path: str, meshfile: str, ndims: int, order: int, viscous: bool,
               bounds: Dict[str, str], params: Optional[Dict[str, object]] = None) -> str:
    """Write a ZEFR input deck (format of reference ``src/input.cpp:31-461``)."""
    p: Dict[str, object] = {
        "nDims": ndims, "meshfile": meshfile, "order": order, "equation": "EulerNS",
        "viscous": int(viscous), "spt_type": "Legendre", "n_steps": 1, "dt_scheme": "RK44",
        "dt_type": 0, "dt": 1e-3, "output_prefix": "zr_out", "write_freq": 0, "report_freq": 0,
        "res_type": 1, "force_freq": 0, "error_freq": 0, "fconv_type": "Rusanov", "fvisc_type": "LDG",
        "rus_k": 0.0, "ldg_b": 0.5, "ldg_tau": 1.0, "ic_type": 0, "gamma": 1.4, "rho_fs": 1.0,
        "P_fs": 1.0, "mach_fs": 0.2,
    }
    if params:
        p.update(params)
    lines = [f"{k} {v}" for k, v in p.items()]
    lines.append("mesh_bound fluid fluid")
    for mesh_name, bc in bounds.items():
        lines.append(f"mesh_bound {mesh_name.lower()} {bc}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
