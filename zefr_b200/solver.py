"""Host-side mirror of ZEFR's FRSolver for the DFR residual path.

Method names follow the reference ``FRSolver`` (include/solver.hpp:140-190):
``compute_residual(stage)`` fills the stage's ``divF_spts`` register,
``update()`` advances one explicit RK44 step, ``step_RK_stage(stage)`` does one
stage, and the state is read and written in the reference layout
``U_spts[spt][var][ele]`` (``get_q_spts`` strides, src/zefr.cpp:607-645).
Everything runs in ``libzefr_b200.so`` on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Union

import numpy as np

from . import _lib
from ._lib import ZbInfo, ZbMesh, ZbParams, check, lib
from .meshgen import Mesh, read_gmsh

_DP = ctypes.POINTER(ctypes.c_double)


def make_params(order: int, viscous: bool = False, *, gamma: float = 1.4, prandtl: float = 0.72, mu: float = 0.0,
                rt: float = 0.0, c_sth: float = 0.0, fix_vis: bool = True, rus_k: float = 0.0,
                ldg_b: float = 0.5, ldg_tau: float = 1.0, rho_fs: float = 1.0, V_fs=(0.0, 0.0, 0.0),
                P_fs: float = 1.0, T_wall: float = 0.0, R_ref: float = 0.0, V_wall=(0.0, 0.0, 0.0),
                dt: float = 1e-3, fconv: str = "rusanov", precision: str = "fp64",
                tensor_ops: bool = False) -> ZbParams:
    """Solver parameters with the meaning of the reference InputStruct fields.
    ``tensor_ops``: mixed form on triangles (Navier-Stokes), the gradient
    kernel's operator products on the tensor pipe (TF32x3)."""
    p = ZbParams()
    p.order = order
    p.viscous = int(bool(viscous))
    p.fconv = {"rusanov": _lib.ZB_FLUX_RUSANOV, "roe": _lib.ZB_FLUX_ROE}[fconv.lower()]
    p.precision = {"fp64": _lib.ZB_FP64, "mixed": _lib.ZB_MIXED}[precision.lower()]
    p.gamma, p.prandtl, p.mu, p.rt, p.c_sth = gamma, prandtl, mu, rt, c_sth
    p.fix_vis = int(bool(fix_vis))
    p.rus_k, p.ldg_b, p.ldg_tau = rus_k, ldg_b, ldg_tau
    p.rho_fs, p.P_fs, p.T_wall, p.R_ref, p.dt = rho_fs, P_fs, T_wall, R_ref, dt
    for d in range(3):
        p.V_fs[d] = float(V_fs[d]) if d < len(V_fs) else 0.0
        p.V_wall[d] = float(V_wall[d]) if d < len(V_wall) else 0.0
    p.tensor_ops = int(bool(tensor_ops))
    return p


def params_from_reference(ref_params: Dict[str, float], order: int, **overrides) -> ZbParams:
    """Build parameters from the reference's InputStruct values (as the oracle reports them)."""
    rp = ref_params
    kw = dict(gamma=rp["gamma"], prandtl=rp["prandtl"], mu=rp["mu"], rt=rp["rt"], c_sth=rp["c_sth"],
              fix_vis=bool(rp["fix_vis"]), rus_k=rp["rus_k"], ldg_b=rp["ldg_b"], ldg_tau=rp["ldg_tau"],
              rho_fs=rp["rho_fs"], V_fs=(rp["V_fs0"], rp["V_fs1"], rp["V_fs2"]), P_fs=rp["P_fs"],
              T_wall=rp["T_wall"], R_ref=rp["R_ref"], V_wall=(rp["V_wall0"], rp["V_wall1"], rp["V_wall2"]),
              dt=rp["dt"])
    kw.update(overrides)
    return make_params(order, bool(rp["viscous"]), **kw)


def params_from_deck(**deck) -> ZbParams:
    """Reference deck keys -> parameters (non-dimensionalisation of src/input.cpp:463-539)."""
    d = _lib.ZbDeck()
    defaults = dict(ndims=2, order=3, viscous=0, fconv=0, precision=0, disable_nondim=0, fix_vis=0, gamma=1.4,
                    prandtl=0.72, R=286.9, S=120.0, T_gas=291.15, rho_fs=1.4, P_fs=1.0, mach_fs=0.2, Re_fs=200.0,
                    L_fs=1.0, T_fs=300.0, nx_fs=1.0, ny_fs=0.0, nz_fs=0.0, mach_wall=0.0, T_wall=300.0,
                    nx_wall=1.0, ny_wall=0.0, nz_wall=0.0, rus_k=0.0, ldg_b=0.5, ldg_tau=1.0, dt=1e-3)
    defaults.update(deck)
    for k, v in defaults.items():
        setattr(d, k, v)
    p = ZbParams()
    check(lib().zb_params_from_deck(ctypes.byref(d), ctypes.byref(p)))
    return p


class _MeshArrays:
    """Keeps numpy buffers alive behind a ZbMesh view."""

    def __init__(self, mesh: Mesh, bounds: Dict[str, str]):
        self.coords = np.ascontiguousarray(mesh.nodes, dtype=np.float64)
        self.ele2nodes = np.ascontiguousarray(mesh.elements, dtype=np.int64)
        npf = max((len(f[1]) for f in mesh.bnd_faces), default=1)
        fn = np.full((max(len(mesh.bnd_faces), 1), npf), -1, dtype=np.int64)
        bc = np.zeros(max(len(mesh.bnd_faces), 1), dtype=np.int32)
        lower = {k.lower(): v.lower() for k, v in bounds.items()}
        for i, (_, nodes, name) in enumerate(mesh.bnd_faces):
            fn[i, :len(nodes)] = nodes
            key = name.lower()
            if key not in lower:
                raise ValueError(f'Unrecognized mesh boundary: "{key}"')
            bc[i] = _lib.BC_CODES[lower[key]]
        self.face_nodes, self.face_bc = fn, bc
        m = ZbMesh()
        m.ndims = mesh.ndims
        m.gmsh_type = mesh.gmsh_type
        m.n_nodes = self.coords.shape[0]
        m.coords = self.coords.ctypes.data_as(_DP)
        m.n_eles = self.ele2nodes.shape[0]
        m.nodes_per_ele = self.ele2nodes.shape[1]
        m.ele2nodes = self.ele2nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        m.n_bnd_faces = len(mesh.bnd_faces)
        m.nodes_per_face = npf
        m.face_nodes = self.face_nodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        m.face_bc = self.face_bc.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        self.view = m


def _as_mesh(mesh: Union[Mesh, str]) -> Mesh:
    return read_gmsh(mesh) if isinstance(mesh, str) else mesh


class Plan:
    """Host-only set-up (connectivity, operators, metrics); needs no GPU."""

    def __init__(self, mesh: Union[Mesh, str], params: ZbParams, bounds: Dict[str, str]):
        mesh = _as_mesh(mesh)
        self._arrays = _MeshArrays(mesh, bounds)
        self._params = params
        h = ctypes.c_void_p()
        check(lib().zb_plan_create(ctypes.byref(self._arrays.view), ctypes.byref(params), ctypes.byref(h)))
        self.h = h
        self.info = ZbInfo()
        check(lib().zb_plan_info(self.h, ctypes.byref(self.info)))

    def get(self, name: str) -> np.ndarray:
        n = ctypes.c_int64(0)
        check(lib().zb_plan_get(self.h, name.encode(), None, ctypes.byref(n)))
        out = np.empty(n.value)
        check(lib().zb_plan_get(self.h, name.encode(), out.ctypes.data_as(_DP), ctypes.byref(n)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().zb_plan_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FRSolver:
    """DFR residual and RK44 stepping on the GPU, FRSolver-style.

    ``mesh`` is a :class:`zefr_b200.meshgen.Mesh` or a gmsh 2.2 file path;
    ``bounds`` maps the mesh's boundary names to deck condition names
    (the deck's ``mesh_bound`` lines, e.g. ``{"PERIODIC": "periodic"}``).
    """

    def __init__(self, mesh: Union[Mesh, str], params: ZbParams, bounds: Dict[str, str]):
        self.plan = Plan(mesh, params, bounds)
        h = ctypes.c_void_p()
        check(lib().zb_create(self.plan.h, ctypes.byref(h)))
        self.h = h
        self.info = ZbInfo()
        check(lib().zb_info_get(self.h, ctypes.byref(self.info)))
        self.nspts, self.nvars, self.neles = self.info.nspts, self.info.nvars, int(self.info.n_eles)
        self.ndims, self.nstages = self.info.ndims, self.info.nstages
        self._stream = None  # caller stream given to set_stream

    # -- lifetime --
    @classmethod
    def from_deck(cls, path: str, precision: str = "fp64") -> "FRSolver":
        """Solver for a reference input deck (mesh file, parameters, mesh_bound
        lines, time scheme; see ``zefr_b200.deck``)."""
        from .deck import read_deck
        d = read_deck(path)
        p = params_from_deck(precision={"fp64": 0, "mixed": 1}[precision], **d.params)
        s = cls(d.meshfile, p, d.bounds)
        if d.dt_scheme != "RK44" or d.time_scheme:
            s.set_time_scheme(d.dt_scheme, **d.time_scheme)
        return s

    def close(self):
        if getattr(self, "h", None):
            lib().zb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def state_shape(self):
        return (self.nspts, self.nvars, self.neles)

    def _strides(self):
        E = self.neles
        return (self.nvars * E, E, 1)

    # -- state --
    def _torch_ready(self):
        """The library runs on its own stream: wait for torch's queued work
        on a tensor before the library reads it (nothing to wait for when the
        library was put on torch's current stream with set_stream)."""
        import torch
        if not self._on_torch_stream():
            torch.cuda.current_stream().synchronize()

    def _on_torch_stream(self) -> bool:
        if self._stream is None:
            return False
        import torch
        return self._stream == torch.cuda.current_stream().cuda_stream

    def _device_done(self) -> None:
        """Device outputs complete for torch: a full wait only when the
        library and torch use different streams."""
        if not self._on_torch_stream():
            self.synchronize()

    def set_state(self, U) -> None:
        if hasattr(U, "is_cuda") and U.is_cuda:
            import torch
            U = U.to(torch.float64).contiguous()
            self._torch_ready()
            assert tuple(U.shape) == self.state_shape
            check(lib().zb_set_state(self.h, ctypes.cast(U.data_ptr(), _DP), *self._strides(), _lib.ZB_DEVICE))
            self._keep = U
            return
        U = np.ascontiguousarray(U, dtype=np.float64)
        if U.shape != self.state_shape:
            raise ValueError(f"state shape {U.shape} != {self.state_shape}")
        check(lib().zb_set_state(self.h, U.ctypes.data_as(_DP), *self._strides(), _lib.ZB_HOST))

    def get_state(self) -> np.ndarray:
        out = np.zeros(self.state_shape)
        check(lib().zb_get_state(self.h, out.ctypes.data_as(_DP), *self._strides(), _lib.ZB_HOST))
        return out

    def get_state_device(self, out) -> None:
        """Copy the state into a contiguous float64 CUDA tensor of state_shape
        (complete on return)."""
        check(lib().zb_get_state(self.h, ctypes.cast(out.data_ptr(), _DP), *self._strides(), _lib.ZB_DEVICE))
        self._device_done()

    # -- residual --
    def compute_residual(self, stage: int = 0) -> None:
        check(lib().zb_compute_residual(self.h, stage))

    # FRSolver::compute_residual_start / _mid / _finish: the three together
    # equal compute_residual (start: flux-point traces; mid: gradient, fluxes
    # and volume divergence for Navier-Stokes; finish: common fluxes and the
    # surface correction)
    def compute_residual_start(self, stage: int = 0) -> None:
        check(lib().zb_compute_residual_start(self.h, stage))

    def compute_residual_mid(self, stage: int = 0) -> None:
        check(lib().zb_compute_residual_mid(self.h, stage))

    def compute_residual_finish(self, stage: int = 0) -> None:
        check(lib().zb_compute_residual_finish(self.h, stage))

    def get_residual(self, stage: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.state_shape)
        elif out.shape != self.state_shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of state_shape")
        check(lib().zb_get_residual(self.h, stage, out.ctypes.data_as(_DP), *self._strides(), _lib.ZB_HOST))
        return out

    def residuals_host(self, states, outs, stage: int = 0) -> None:
        """divF(stage) of each host state into the matching host array
        (zb_compute_residuals_host): C-contiguous float64 arrays of
        state_shape; pinned memory (e.g. numpy views of pinned torch tensors)
        lets the copies overlap the computation."""
        if len(states) != len(outs):
            raise ValueError("states and outputs differ in number")
        for a in list(states) + list(outs):
            if a.shape != self.state_shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("arrays must be C-contiguous float64 of state_shape")
        n = len(states)
        U = (_DP * n)(*[a.ctypes.data_as(_DP) for a in states])
        R = (_DP * n)(*[a.ctypes.data_as(_DP) for a in outs])
        check(lib().zb_compute_residuals_host(self.h, stage, n, U, R))

    def get_residual_device(self, out, stage: int = 0) -> None:
        """Copy a residual register into a contiguous float64 CUDA tensor
        (complete on return)."""
        check(lib().zb_get_residual(self.h, stage, ctypes.cast(out.data_ptr(), _DP), *self._strides(),
                                    _lib.ZB_DEVICE))
        self._device_done()

    def residual(self, U, stage: int = 0) -> np.ndarray:
        self.set_state(U)
        self.compute_residual(stage)
        return self.get_residual(stage)

    # -- time stepping --
    def step_RK_stage(self, stage: int) -> None:
        check(lib().zb_rk_stage(self.h, stage))

    # FRSolver::step_RK_stage_start / _mid / _finish (the RK update in finish)
    def step_RK_stage_start(self, stage: int) -> None:
        check(lib().zb_rk_stage_start(self.h, stage))

    def step_RK_stage_mid(self, stage: int) -> None:
        check(lib().zb_rk_stage_mid(self.h, stage))

    def step_RK_stage_finish(self, stage: int) -> None:
        check(lib().zb_rk_stage_finish(self.h, stage))

    def update(self) -> None:
        check(lib().zb_step(self.h, 1))

    def step(self, n: int) -> None:
        check(lib().zb_step(self.h, n))

    def set_dt(self, dt: float) -> None:
        check(lib().zb_set_dt(self.h, dt))

    def set_time_scheme(self, dt_scheme: str = "RK44", **kw) -> None:
        """Time integration with the reference deck's keys (src/input.cpp:72-127):
        ``dt_scheme`` "RK44" or "RK54"; ``dt_type`` 0/1/2, ``CFL``, ``CFL_type``;
        ``adapt_dt`` and ``err_atol``, ``err_rtol``, ``pi_alpha``, ``pi_beta``,
        ``safety_factor``, ``max_factor``, ``min_factor``, ``max_dt``.  Keys not
        given keep the deck defaults."""
        ts = _lib.ZbTimeScheme()
        lib().zb_time_scheme_defaults(ctypes.byref(ts))
        schemes = {"RK44": _lib.ZB_RK44, "RK54": _lib.ZB_RK54}
        if dt_scheme not in schemes:
            raise ValueError(f"dt_scheme must be one of {sorted(schemes)}")
        ts.scheme = schemes[dt_scheme]
        keys = {"dt_type": "dt_type", "CFL": "cfl", "CFL_type": "cfl_type", "adapt_dt": "adapt_dt",
                "err_atol": "atol", "err_rtol": "rtol", "pi_alpha": "pi_alpha", "pi_beta": "pi_beta",
                "safety_factor": "safety", "max_factor": "max_factor", "min_factor": "min_factor", "max_dt": "max_dt"}
        for k, v in kw.items():
            if k not in keys:
                raise ValueError(f"unknown time-scheme key {k!r}")
            setattr(ts, keys[k], type(getattr(ts, keys[k]))(v))
        check(lib().zb_set_time_scheme(self.h, ctypes.byref(ts)))

    def time_state(self) -> Dict[str, float]:
        """dt the next step starts from, last accepted error estimate, rejected
        steps and flow time."""
        dt, err, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rej = ctypes.c_int64()
        check(lib().zb_time_state(self.h, ctypes.byref(dt), ctypes.byref(err), ctypes.byref(rej), ctypes.byref(t)))
        return {"dt": dt.value, "prev_err": err.value, "rejected": int(rej.value), "flow_time": t.value}

    def element_dt(self) -> np.ndarray:
        """Per-element step of the last CFL estimate, [n_eles]."""
        out = np.zeros(self.info.n_eles)
        check(lib().zb_get_element_dt(self.h, out.ctypes.data_as(_DP)))
        return out

    def set_freestream(self, rho_fs: float, V_fs, P_fs: float) -> None:
        """Free-stream state of the far-field / characteristic boundaries."""
        v = np.zeros(3)
        v[:len(V_fs)] = V_fs
        check(lib().zb_set_freestream(self.h, float(rho_fs), v.ctypes.data_as(_DP), float(P_fs)))

    def residual_norms(self) -> Dict[str, np.ndarray]:
        out = np.zeros(3 * self.nvars)
        check(lib().zb_residual_norms(self.h, out.ctypes.data_as(_DP)))
        V = self.nvars
        return {"linf": out[:V], "l1": out[V:2 * V], "l2": out[2 * V:]}

    def functionals(self) -> Dict[str, float]:
        """FP64 volume integrals of the current state (report_turbulent_stats):
        kinetic energy, enstrophy (Navier-Stokes) and volume."""
        out = np.zeros(4)
        check(lib().zb_functionals(self.h, out.ctypes.data_as(_DP)))
        return {"ke": float(out[0]), "enstrophy": float(out[1]), "volume": float(out[2])}

    # -- adjoint --
    def vjp(self, lam, params: bool = False):
        """Adjoint of the residual at the current state (plain FP64 form):
        returns Ubar = (d divF / d U)^T lam in state_shape, and with
        ``params`` also d(lam . divF)/d(rho_fs, V_fs[0..2], P_fs).  ``lam``
        is a numpy array or a CUDA tensor (then Ubar is a CUDA tensor)."""
        pbar = np.zeros(5) if params else None
        pptr = pbar.ctypes.data_as(_DP) if params else None
        if hasattr(lam, "is_cuda") and lam.is_cuda:
            import torch
            lam = lam.to(torch.float64).contiguous()
            assert tuple(lam.shape) == self.state_shape
            out = torch.empty_like(lam)
            self._torch_ready()
            check(lib().zb_vjp(self.h, ctypes.cast(lam.data_ptr(), _DP), ctypes.cast(out.data_ptr(), _DP),
                               *self._strides(), _lib.ZB_DEVICE, pptr))
            self._device_done()
        else:
            lam = np.ascontiguousarray(lam, dtype=np.float64)
            if lam.shape != self.state_shape:
                raise ValueError(f"lam shape {lam.shape} != {self.state_shape}")
            out = np.zeros(self.state_shape)
            check(lib().zb_vjp(self.h, lam.ctypes.data_as(_DP), out.ctypes.data_as(_DP), *self._strides(),
                               _lib.ZB_HOST, pptr))
        return (out, pbar) if params else out

    def wall_force(self) -> Dict[str, np.ndarray]:
        """FP64 force and moment (about the origin) on the wall boundaries
        (compute_moments) of the current state."""
        out = np.zeros(6)
        check(lib().zb_wall_force(self.h, out.ctypes.data_as(_DP)))
        return {"force": out[:3].copy(), "moment": out[3:].copy()}

    def vjp_geometry(self, lam):
        """Adjoint of the residual at the current state with respect to the
        state, the free-stream state and the geometry (plain FP64 form, host
        arrays): returns (Ubar, pbar, {"inv_jaco": [D,S,D,E], "jaco_det":
        [S,E], "norm": [Fp,D,E], "dA": [Fp,E]})."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        if lam.shape != self.state_shape:
            raise ValueError(f"lam shape {lam.shape} != {self.state_shape}")
        S, V, E = self.state_shape
        D, Fp = self.ndims, self.info.nfpts
        out = np.zeros(self.state_shape)
        pbar = np.zeros(5)
        g = {"inv_jaco": np.zeros((D, S, D, E)), "jaco_det": np.zeros((S, E)), "norm": np.zeros((Fp, D, E)),
             "dA": np.zeros((Fp, E))}
        check(lib().zb_vjp_geometry(self.h, lam.ctypes.data_as(_DP), out.ctypes.data_as(_DP), *self._strides(),
                                    _lib.ZB_HOST, pbar.ctypes.data_as(_DP), g["inv_jaco"].ctypes.data_as(_DP),
                                    g["jaco_det"].ctypes.data_as(_DP), g["norm"].ctypes.data_as(_DP),
                                    g["dA"].ctypes.data_as(_DP)))
        return out, pbar, g

    def vjp_geometry_accumulate(self, lam):
        """``vjp(lam, params=True)`` on a CUDA tensor that also adds the
        geometry adjoint to device-side sums (read with
        :meth:`geometry_adjoint`)."""
        import torch
        lam = lam.to(torch.float64).contiguous()
        assert tuple(lam.shape) == self.state_shape
        out = torch.empty_like(lam)
        pbar = np.zeros(5)
        self._torch_ready()
        check(lib().zb_vjp_geometry_accumulate(self.h, ctypes.cast(lam.data_ptr(), _DP),
                                               ctypes.cast(out.data_ptr(), _DP), *self._strides(), _lib.ZB_DEVICE,
                                               pbar.ctypes.data_as(_DP)))
        self._device_done()
        return out, pbar

    def rk_step_vjp(self, U0, Ubar1, pbar: Optional[np.ndarray] = None, geometry: bool = False):
        """Reverse of one RK44 step from U0 (CUDA tensors of state_shape):
        returns (dU1/dU0)^T Ubar1, adds the free-stream adjoint to ``pbar``
        (5 values) and, with ``geometry``, the metric adjoint to the
        device-side sums of :meth:`geometry_adjoint`.  Stage states and
        residuals are recomputed in the library (zb_rk_step_vjp)."""
        import torch
        U0 = U0.to(torch.float64).contiguous()
        Ubar1 = Ubar1.to(torch.float64).contiguous()
        assert tuple(U0.shape) == self.state_shape and tuple(Ubar1.shape) == self.state_shape
        out = torch.empty_like(U0)
        p = np.zeros(5)
        self._torch_ready()
        check(lib().zb_rk_step_vjp(self.h, ctypes.cast(U0.data_ptr(), _DP), ctypes.cast(Ubar1.data_ptr(), _DP),
                                   ctypes.cast(out.data_ptr(), _DP), *self._strides(), _lib.ZB_DEVICE,
                                   p.ctypes.data_as(_DP), 1 if geometry else 0))
        self._device_done()
        if pbar is not None:
            pbar += p
        return out

    def geometry_adjoint(self, reset: bool = True) -> Dict[str, np.ndarray]:
        """The summed geometry adjoint of vjp_geometry_accumulate (host arrays)."""
        S, V, E = self.state_shape
        D, Fp = self.ndims, self.info.nfpts
        g = {"inv_jaco": np.zeros((D, S, D, E)), "jaco_det": np.zeros((S, E)), "norm": np.zeros((Fp, D, E)),
             "dA": np.zeros((Fp, E))}
        check(lib().zb_geometry_adjoint_get(self.h, g["inv_jaco"].ctypes.data_as(_DP),
                                            g["jaco_det"].ctypes.data_as(_DP), g["norm"].ctypes.data_as(_DP),
                                            g["dA"].ctypes.data_as(_DP), 1 if reset else 0))
        return g

    # -- geometry from element nodes (zb_geometry_eval, zb_set_nodes) --
    @property
    def nodes_shape(self):
        """(nNodes, ndims, neles): the element node layout Elements::nodes."""
        if getattr(self, "_nodes_shape", None) is None:
            n = self.plan.get("nodes").size
            self._nodes_shape = (n // (self.ndims * self.neles), self.ndims, self.neles)
        return self._nodes_shape

    def _geometry_shapes(self):
        S, D, E, Fp = self.nspts, self.ndims, self.neles, self.info.nfpts
        return {"inv_jaco": (D, S, D, E), "jaco_det": (S, E), "norm": (Fp, D, E), "dA": (Fp, E)}

    def geometry_eval(self, nodes):
        """Set-up metrics of element nodes [nNodes][D][E] (float64 CUDA
        tensor), computed on the device by zb_geometry_eval: a dict of CUDA
        tensors inv_jaco [D,S,D,E], jaco_det [S,E], norm [Fp,D,E], dA [Fp,E]."""
        import torch
        nodes = nodes.to(torch.float64).contiguous()
        if tuple(nodes.shape) != self.nodes_shape or not nodes.is_cuda:
            raise ValueError(f"nodes must be a CUDA tensor of shape {self.nodes_shape}")
        out = {k: torch.empty(s, dtype=torch.float64, device=nodes.device) for k, s in self._geometry_shapes().items()}
        self._torch_ready()
        check(lib().zb_geometry_eval(self.h, ctypes.cast(nodes.data_ptr(), _DP),
                                     *(ctypes.cast(out[k].data_ptr(), _DP) for k in ("inv_jaco", "jaco_det", "norm", "dA")),
                                     _lib.ZB_DEVICE))
        self._device_done()
        return out

    def geometry_eval_vjp(self, nodes, bars: Dict[str, object]):
        """Adjoint of :meth:`geometry_eval` at ``nodes``: the node adjoint
        [nNodes][D][E] (CUDA tensor) of metric adjoints ``bars`` (keys as
        geometry_eval's; missing keys count as zero)."""
        import torch
        nodes = nodes.to(torch.float64).contiguous()
        if tuple(nodes.shape) != self.nodes_shape or not nodes.is_cuda:
            raise ValueError(f"nodes must be a CUDA tensor of shape {self.nodes_shape}")
        shapes = self._geometry_shapes()
        held, ptrs = [], []
        for k in ("inv_jaco", "jaco_det", "norm", "dA"):
            b = bars.get(k)
            if b is None:
                ptrs.append(None)
                continue
            b = torch.as_tensor(b, dtype=torch.float64, device=nodes.device).contiguous()
            if tuple(b.shape) != shapes[k]:
                raise ValueError(f"{k} adjoint must have shape {shapes[k]}")
            held.append(b)
            ptrs.append(ctypes.cast(b.data_ptr(), _DP))
        out = torch.empty_like(nodes)
        self._torch_ready()
        check(lib().zb_geometry_eval_vjp(self.h, ctypes.cast(nodes.data_ptr(), _DP), *ptrs,
                                         ctypes.cast(out.data_ptr(), _DP), _lib.ZB_DEVICE))
        self._device_done()
        return out

    def set_nodes(self, nodes) -> None:
        """Move the mesh (zb_set_nodes): new element nodes [nNodes][D][E], a
        numpy array or a CUDA tensor; metrics are recomputed on the device."""
        if hasattr(nodes, "is_cuda") and nodes.is_cuda:
            import torch
            nodes = nodes.to(torch.float64).contiguous()
            if tuple(nodes.shape) != self.nodes_shape:
                raise ValueError(f"nodes must have shape {self.nodes_shape}")
            self._torch_ready()
            check(lib().zb_set_nodes(self.h, ctypes.cast(nodes.data_ptr(), _DP), _lib.ZB_DEVICE))
            self._device_done()
        else:
            nodes = np.ascontiguousarray(nodes, dtype=np.float64)
            if nodes.shape != self.nodes_shape:
                raise ValueError(f"nodes must have shape {self.nodes_shape}")
            check(lib().zb_set_nodes(self.h, nodes.ctypes.data_as(_DP), _lib.ZB_HOST))

    def set_stream(self, stream_ptr: int) -> None:
        check(lib().zb_set_stream(self.h, ctypes.c_void_p(stream_ptr)))
        self._stream = stream_ptr

    def synchronize(self) -> None:
        check(lib().zb_synchronize(self.h))

    def launch_count(self) -> int:
        return int(lib().zb_launch_count(self.h))

    def profile(self, on: bool = True) -> None:
        """Record CUDA events around every kernel launch (device timing per kernel)."""
        check(lib().zb_profile_enable(self.h, int(on)))

    def profile_read(self) -> Dict[str, tuple]:
        """{kernel name: (total ms, launches)} since the last read."""
        ms = np.zeros(_lib.ZB_NKERNELS)
        cnt = np.zeros(_lib.ZB_NKERNELS, dtype=np.int64)
        check(lib().zb_profile_read(self.h, ms.ctypes.data_as(_DP), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return {lib().zb_kernel_name(k).decode(): (float(ms[k]), int(cnt[k])) for k in range(_lib.ZB_NKERNELS)
                if cnt[k] > 0}
