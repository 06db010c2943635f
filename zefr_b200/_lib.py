"""ctypes binding of the C ABI in ``include/zb.h`` (libzefr_b200.so).

The library is built in-tree by ``zefr_b200/csrc/Makefile``; importing this
module without it raises immediately -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzefr_b200.so")

# status codes (zb.h)
ZB_OK = 0
STATUS_NAMES = {0: "ZB_OK", -1: "ZB_ERR_ARG", -2: "ZB_ERR_CUDA", -3: "ZB_ERR_MESH", -4: "ZB_ERR_UNSUPPORTED",
                -5: "ZB_ERR_NONFINITE", -6: "ZB_ERR_NOMEM", -7: "ZB_ERR_INTERNAL"}
ZB_FP64, ZB_MIXED = 0, 1
ZB_HOST, ZB_DEVICE = 0, 1
ZB_FLUX_RUSANOV, ZB_FLUX_ROE = 0, 2

# Deck boundary names -> condition codes (reference src/input.cpp:12-29)
BC_CODES = {
    "none": 0, "fluid": 0, "periodic": 1, "char": 2, "farfield": 3, "inlet_sup": 3, "outlet_sup": 4,
    "wall_slip": 5, "wall_ns_iso": 6, "wall_ns_adi": 7, "wall_ns_iso_move": 8, "wall_ns_adi_move": 9,
    "symmetry": 11,
}

EXPORTED = [
    "zb_last_error", "zb_version", "zb_params_from_deck", "zb_mesh_read_gmsh", "zb_mesh_free",
    "zb_plan_create", "zb_plan_free", "zb_plan_info", "zb_plan_get", "zb_create", "zb_create_from_mesh",
    "zb_destroy", "zb_info_get", "zb_set_stream", "zb_set_dt", "zb_set_state", "zb_get_state",
    "zb_compute_residual", "zb_get_residual", "zb_rk_stage", "zb_step", "zb_residual_norms",
    "zb_synchronize", "zb_launch_count", "zb_profile_enable", "zb_profile_read", "zb_kernel_name",
    "zb_compute_residual_noalloc", "zb_functionals", "zb_vjp", "zb_set_freestream", "zb_wall_force", "zb_vjp_geometry",
    "zb_vjp_geometry_accumulate", "zb_geometry_adjoint_get",
    "zb_batch_create", "zb_batch_destroy", "zb_batch_autotune", "zb_batch_autotune_form", "zb_batch_set_config",
    "zb_batch_step",
    "zb_batch_stage", "zb_batch_synchronize", "zb_batch_launch_count",
    "zb_time_scheme_defaults", "zb_set_time_scheme", "zb_time_state", "zb_get_element_dt", "zb_rk_step_vjp",
    "zb_geometry_eval", "zb_geometry_eval_vjp", "zb_set_nodes",
    "zb_compute_residual_start", "zb_compute_residual_mid", "zb_compute_residual_finish",
    "zb_rk_stage_start", "zb_rk_stage_mid", "zb_rk_stage_finish", "zb_operator_mm_tf32x3",
    "zb_compute_residuals_host",
]
ZB_RK44, ZB_RK54 = 0, 1
ZB_NKERNELS = 11


class ZbMesh(ctypes.Structure):
    _fields_ = [
        ("ndims", ctypes.c_int), ("gmsh_type", ctypes.c_int), ("n_nodes", ctypes.c_int64),
        ("coords", ctypes.POINTER(ctypes.c_double)), ("n_eles", ctypes.c_int64), ("nodes_per_ele", ctypes.c_int),
        ("ele2nodes", ctypes.POINTER(ctypes.c_int64)), ("n_bnd_faces", ctypes.c_int64),
        ("nodes_per_face", ctypes.c_int), ("face_nodes", ctypes.POINTER(ctypes.c_int64)),
        ("face_bc", ctypes.POINTER(ctypes.c_int)),
    ]


class ZbParams(ctypes.Structure):
    _fields_ = [
        ("order", ctypes.c_int), ("viscous", ctypes.c_int), ("fconv", ctypes.c_int), ("precision", ctypes.c_int),
        ("gamma", ctypes.c_double), ("prandtl", ctypes.c_double), ("mu", ctypes.c_double), ("rt", ctypes.c_double),
        ("c_sth", ctypes.c_double), ("fix_vis", ctypes.c_int), ("rus_k", ctypes.c_double),
        ("ldg_b", ctypes.c_double), ("ldg_tau", ctypes.c_double), ("rho_fs", ctypes.c_double),
        ("V_fs", ctypes.c_double * 3), ("P_fs", ctypes.c_double), ("T_wall", ctypes.c_double),
        ("R_ref", ctypes.c_double), ("V_wall", ctypes.c_double * 3), ("dt", ctypes.c_double),
        ("tri_volume_div", ctypes.c_int), ("tensor_ops", ctypes.c_int),
    ]


class ZbTimeScheme(ctypes.Structure):
    _fields_ = [
        ("scheme", ctypes.c_int), ("dt_type", ctypes.c_int), ("cfl_type", ctypes.c_int), ("cfl", ctypes.c_double),
        ("adapt_dt", ctypes.c_int), ("atol", ctypes.c_double), ("rtol", ctypes.c_double),
        ("pi_alpha", ctypes.c_double), ("pi_beta", ctypes.c_double), ("safety", ctypes.c_double),
        ("max_factor", ctypes.c_double), ("min_factor", ctypes.c_double), ("max_dt", ctypes.c_double),
    ]


class ZbBatchConfig(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("blocks_per_sm", ctypes.c_int), ("order", ctypes.c_int),
                ("ms_per_step", ctypes.c_double), ("group", ctypes.c_int), ("chunk", ctypes.c_int),
                ("fused", ctypes.c_int)]


class ZbDeck(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("ndims", "order", "viscous", "fconv", "precision", "disable_nondim",
                                            "fix_vis")] + \
               [(n, ctypes.c_double) for n in ("gamma", "prandtl", "R", "S", "T_gas", "rho_fs", "P_fs", "mach_fs",
                                               "Re_fs", "L_fs", "T_fs", "nx_fs", "ny_fs", "nz_fs", "mach_wall",
                                               "T_wall", "nx_wall", "ny_wall", "nz_wall", "rus_k", "ldg_b",
                                               "ldg_tau", "dt")]


class ZbInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("ndims", "nvars", "nspts", "nfpts", "order", "etype")] + \
               [(n, ctypes.c_int64) for n in ("n_eles", "n_eles_pad", "n_gfpts", "n_gfpts_int", "n_gfpts_bnd")] + \
               [(n, ctypes.c_int) for n in ("nstages", "tile", "precision")]


class ZbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `make -C zefr_b200/csrc` "
                              "(the residual has no CPU implementation)")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, i64 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64
        L.zb_last_error.restype = ctypes.c_char_p
        L.zb_version.restype = ctypes.c_char_p
        L.zb_params_from_deck.argtypes = [ctypes.POINTER(ZbDeck), ctypes.POINTER(ZbParams)]
        L.zb_mesh_read_gmsh.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.POINTER(ZbMesh))]
        L.zb_mesh_free.argtypes = [ctypes.POINTER(ZbMesh)]
        L.zb_mesh_free.restype = None
        L.zb_plan_create.argtypes = [ctypes.POINTER(ZbMesh), ctypes.POINTER(ZbParams), ctypes.POINTER(vp)]
        L.zb_plan_free.argtypes = [vp]
        L.zb_plan_free.restype = None
        L.zb_plan_info.argtypes = [vp, ctypes.POINTER(ZbInfo)]
        L.zb_plan_get.argtypes = [vp, ctypes.c_char_p, dp, ctypes.POINTER(i64)]
        L.zb_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.zb_create_from_mesh.argtypes = [ctypes.POINTER(ZbMesh), ctypes.POINTER(ZbParams), ctypes.POINTER(vp)]
        L.zb_destroy.argtypes = [vp]
        L.zb_destroy.restype = None
        L.zb_info_get.argtypes = [vp, ctypes.POINTER(ZbInfo)]
        L.zb_set_stream.argtypes = [vp, vp]
        L.zb_set_dt.argtypes = [vp, ctypes.c_double]
        L.zb_set_state.argtypes = [vp, dp, i64, i64, i64, ctypes.c_int]
        L.zb_get_state.argtypes = [vp, dp, i64, i64, i64, ctypes.c_int]
        L.zb_compute_residual.argtypes = [vp, ctypes.c_uint]
        L.zb_get_residual.argtypes = [vp, ctypes.c_uint, dp, i64, i64, i64, ctypes.c_int]
        L.zb_rk_stage.argtypes = [vp, ctypes.c_uint]
        L.zb_compute_residuals_host.argtypes = [vp, ctypes.c_uint, ctypes.c_int, ctypes.POINTER(dp),
                                                ctypes.POINTER(dp)]
        fp = ctypes.POINTER(ctypes.c_float)
        L.zb_operator_mm_tf32x3.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, fp,
                                            ctypes.c_int, fp, ctypes.c_int, ctypes.c_float, fp, ctypes.c_int, vp]
        for fn in ("zb_compute_residual_start", "zb_compute_residual_mid", "zb_compute_residual_finish",
                   "zb_rk_stage_start", "zb_rk_stage_mid", "zb_rk_stage_finish"):
            getattr(L, fn).argtypes = [vp, ctypes.c_uint]
        L.zb_step.argtypes = [vp, ctypes.c_int]
        L.zb_residual_norms.argtypes = [vp, dp]
        L.zb_synchronize.argtypes = [vp]
        L.zb_launch_count.argtypes = [vp]
        L.zb_launch_count.restype = ctypes.c_int64
        L.zb_profile_enable.argtypes = [vp, ctypes.c_int]
        L.zb_profile_read.argtypes = [vp, dp, ctypes.POINTER(i64)]
        L.zb_kernel_name.restype = ctypes.c_char_p
        L.zb_kernel_name.argtypes = [ctypes.c_int]
        L.zb_compute_residual_noalloc.argtypes = [vp, dp, dp, vp]
        L.zb_functionals.argtypes = [vp, dp]
        L.zb_wall_force.argtypes = [vp, dp]
        L.zb_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp)]
        L.zb_batch_destroy.argtypes = [vp]
        L.zb_batch_destroy.restype = None
        L.zb_batch_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ZbBatchConfig)]
        L.zb_batch_autotune_form.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ZbBatchConfig)]
        L.zb_batch_set_config.argtypes = [vp, ctypes.POINTER(ZbBatchConfig)]
        L.zb_batch_step.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.zb_batch_stage.argtypes = [vp, ctypes.c_uint]
        L.zb_batch_synchronize.argtypes = [vp]
        L.zb_batch_launch_count.argtypes = [vp]
        L.zb_batch_launch_count.restype = i64
        L.zb_set_freestream.argtypes = [vp, ctypes.c_double, dp, ctypes.c_double]
        L.zb_vjp.argtypes = [vp, dp, dp, i64, i64, i64, ctypes.c_int, dp]
        L.zb_vjp_geometry_accumulate.argtypes = [vp, dp, dp, i64, i64, i64, ctypes.c_int, dp]
        L.zb_geometry_adjoint_get.argtypes = [vp, dp, dp, dp, dp, ctypes.c_int]
        L.zb_vjp_geometry.argtypes = [vp, dp, dp, i64, i64, i64, ctypes.c_int, dp, dp, dp, dp, dp]
        L.zb_time_scheme_defaults.argtypes = [ctypes.POINTER(ZbTimeScheme)]
        L.zb_time_scheme_defaults.restype = None
        L.zb_set_time_scheme.argtypes = [vp, ctypes.POINTER(ZbTimeScheme)]
        L.zb_time_state.argtypes = [vp, dp, dp, ctypes.POINTER(i64), dp]
        L.zb_get_element_dt.argtypes = [vp, dp]
        L.zb_rk_step_vjp.argtypes = [vp, dp, dp, dp, i64, i64, i64, ctypes.c_int, dp, ctypes.c_int]
        L.zb_geometry_eval.argtypes = [vp, dp, dp, dp, dp, dp, ctypes.c_int]
        L.zb_geometry_eval_vjp.argtypes = [vp, dp, dp, dp, dp, dp, dp, ctypes.c_int]
        L.zb_set_nodes.argtypes = [vp, dp, ctypes.c_int]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != ZB_OK:
        raise ZbError(status, lib().zb_last_error().decode())
