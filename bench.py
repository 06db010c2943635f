#!/usr/bin/env python
"""Throughput of the DFR residual on one B200 (or N independent replicas).

Workload: 3D Taylor-Green vortex, 64^3 linear hexes on periodic [0,2pi]^3,
P = 3 (64 solution points per element, 5 conserved variables, 83.9 M DOF),
Re = 1600, Ma = 0.1, Pr = 0.71, Roe convective + LDG viscous flux (beta 0.5,
tau 0.1).  Synthetic: the mesh and the Taylor-Green initial state are
generated in-process.

One step = one residual evaluation FRSolver::compute_residual(stage):
extrapolation to flux points, gradients, fluxes, common fluxes and the
divergence.  Two precision forms are timed: the plain FP64 form (matches the
reference's residual to 1e-12) and the mixed form (FP32 state stored as the
deviation from its mean, FP32 traces, metrics and arithmetic; FP64 set-up and
reductions).  The mixed form is the headline only when its residual is within
1e-5 relative L2 of the FP64 form's on the same state; otherwise value is the
FP64 form's throughput and the mixed form is reported beside it with its
errors (residual on the same input state, residual on the FP32-rounded state,
state after 60 RK44 steps, kinetic-energy and dissipation histories).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NCELL = 64
ORDER = 3
METRIC = "GDOF/s per residual (TGV 64^3 hex P3 NS; mixed form if within 1e-5 of FP64, else FP64)"
WORKLOAD = "taylor_green_64^3_hex_P3_navier_stokes_roe_ldg"
# the reference has no Roe flux: its arm runs the same case with Rusanov on a
# bounded sample of the mesh (per-DOF throughput falls with mesh size on the
# CPU, so a smaller sample flatters the reference)
REF_CELLS = 32
MIXED_GATE = 1e-5
TGV_DECK = dict(ndims=3, order=ORDER, viscous=1, disable_nondim=1, fix_vis=1, mach_fs=0.1, Re_fs=1600.0,
                prandtl=0.71, P_fs=1.0, rho_fs=1.0, L_fs=1.0, ldg_b=0.5, ldg_tau=0.1, dt=5e-4, gamma=1.4)


# DRAM bytes per element of one mixed-form residual (gradient and face
# kernels), read + write, from an ncu capture at 48^3 hexes (state 141 MB,
# above L2): 884.7 + 584.6 MB over 110,592 elements.
MIXED_DRAM_BYTES_PER_ELEMENT = 13286.0
# the same for the FP64 form (k_hex_ns_grad + k_hex_ns_face, FP64, 48^3
# hexes, state 283 MB): 1733.5 + 978.8 MB over 110,592 elements
FP64_DRAM_BYTES_PER_ELEMENT = 24525.0


def b_alg(E: int, S: int, V: int, D: int, G: int, Fp: int, w: int) -> float:
    """Compulsory bytes of one residual: state in + residual out, adjugate + |J|
    at solution points, face normal + two dA per face point, int32 partner +
    int8 slot per element flux point."""
    return E * S * V * (w + w) + E * S * (D * D + 1) * w + G * (D + 2) * w + E * Fp * 5


# ---------------------------------------------------------------------------
# process / timing helpers
# ---------------------------------------------------------------------------

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        with open(self.path) as f:
            out = self.summary(f)
        os.unlink(self.path)
        return out

    @staticmethod
    def summary(lines):
        """Median SM clock, maximum clock, sample count and the throttle
        reasons seen Active, from nvidia-smi CSV lines in FIELDS order."""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def build_solver(precision: str, n: int, flux: str = "roe"):
    import torch
    from zefr_b200 import ics, meshgen
    from zefr_b200.solver import FRSolver, params_from_deck

    mesh = meshgen.box_hexes(n, n, n)
    p = params_from_deck(fconv={"roe": 2, "rusanov": 0}[flux], precision={"fp64": 0, "mixed": 1}[precision],
                         **TGV_DECK)
    s = FRSolver(mesh, p, {"PERIODIC": "periodic"})
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    X = s.plan.get("coord_spts").reshape(s.nspts, 3, s.neles)
    U = ics.taylor_green(X, mach=TGV_DECK["mach_fs"], gamma=TGV_DECK["gamma"])
    return s, U


def barrier_sync(world):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        if torch.cuda.is_available():
            torch.cuda.synchronize()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def time_residuals(s, K: int, W: int, world: int):
    import torch
    for i in range(W):
        s.compute_residual(i % 4)
    barrier_sync(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = s.launch_count()
    e0.record()
    for i in range(K):
        s.compute_residual(i % 4)
    e1.record()
    barrier_sync(world)
    ms = e0.elapsed_time(e1) / K
    return max_over_ranks(ms, world), s.launch_count() - n0


def kernel_profile(s, K: int):
    s.profile(True)
    s.profile_read()
    for i in range(K):
        s.compute_residual(i % 4)
    prof = s.profile_read()
    s.profile(False)
    return {k: {"ms_avg": v[0] / max(v[1], 1), "launches": v[1], "ms_total": v[0]} for k, v in prof.items()}


def time_adjoint(s, U, K: int, W: int):
    """Per-kernel CUDA-event time of one adjoint application (zb_vjp on device
    tensors) at the state U: traces, lift, volume/face pass, trace pass."""
    import torch
    s.set_state(U)
    g = torch.Generator(device="cuda").manual_seed(3)
    lam = torch.randn(s.state_shape, dtype=torch.float64, device="cuda", generator=g)
    for _ in range(max(W, 1)):
        s.vjp(lam)
    s.profile(True)
    s.profile_read()
    for _ in range(K):
        s.vjp(lam)
    prof = s.profile_read()
    s.profile(False)
    names = ("k_extrap", "k_adj_lift", "k_adj_vol", "k_adj_trace")
    kern = {k: {"ms_avg": prof[k][0] / max(prof[k][1], 1), "launches": prof[k][1]} for k in names if prof[k][1]}
    return {"ms_per_vjp": sum(v["ms_avg"] for v in kern.values()), "kernels": kern}


def time_rk_stage(s, K: int, world: int):
    import torch
    for st in range(4):
        s.step_RK_stage(st)
    barrier_sync(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    n = max(4, (K // 4) * 4)
    for i in range(n):
        s.step_RK_stage(i % 4)
    e1.record()
    barrier_sync(world)
    return max_over_ranks(e0.elapsed_time(e1) / n, world)


def time_e2e(s, U, K: int, W: int, world: int):
    """Public API with host buffers: K states in pinned host memory through
    zb_compute_residuals_host, each step copying its state to the device,
    computing the residual and copying it back to pinned host memory (the
    copies of neighbouring steps overlap the computation); host clock around
    the call, which returns with every residual in host memory."""
    import torch
    Uh = [torch.from_numpy(np.ascontiguousarray(U)).pin_memory() for _ in range(2)]
    Rh = [torch.empty_like(Uh[0]).pin_memory() for _ in range(2)]
    Un, Rn = [u.numpy() for u in Uh], [r.numpy() for r in Rh]
    s.residuals_host([Un[i % 2] for i in range(W)], [Rn[i % 2] for i in range(W)], 0)
    barrier_sync(world)
    t0 = time.perf_counter()
    s.residuals_host([Un[i % 2] for i in range(K)], [Rn[i % 2] for i in range(K)], 0)
    barrier_sync(world)
    ms = (time.perf_counter() - t0) * 1e3 / K
    return max_over_ranks(ms, world), Un[0].nbytes, Rn[0].nbytes


def triangle_solver(form: str, mesh=None):
    """Triangle workload: 128 x 128 quads on periodic [0,1]^2 split along seeded
    diagonals (32,768 triangles), interior nodes jittered 15% of h, P4
    (15 Williams-Shunn points), Roe + LDG (beta 0.5, tau 0.1), Ma 0.2, Re 1000,
    Pr 0.71, double shear layer with seeded 1e-3 velocity noise; the solver of
    one form on torch's current stream, with the state set."""
    import torch
    from zefr_b200 import ics, meshgen
    from zefr_b200.solver import FRSolver, params_from_deck
    if mesh is None:
        mesh = meshgen.box_tris(128, seed=2024, jitter=0.15)
    p = params_from_deck(ndims=2, order=4, viscous=1, disable_nondim=1, fix_vis=1, mach_fs=0.2, Re_fs=1000.0,
                         prandtl=0.71, P_fs=1.0, rho_fs=1.0, L_fs=1.0, ldg_b=0.5, ldg_tau=0.1, fconv=2,
                         precision={"mixed": 1, "mixed_tc": 1, "fp64": 0}[form], gamma=1.4, dt=1e-4)
    p.tensor_ops = int(form == "mixed_tc")
    s = FRSolver(mesh, p, {"PERIODIC": "periodic"})
    s.set_stream(torch.cuda.current_stream().cuda_stream)
    X = s.plan.get("coord_spts").reshape(s.nspts, 2, s.neles)
    s.set_state(ics.double_shear_layer(X, mach=0.2, noise=1e-3, seed=7))
    return s


def triangle_side(K: int, W: int):
    """The triangle workload (triangle_solver): GDOF/s per residual of the
    FP64 form and of the mixed form with its gradient kernel's operator
    products on CUDA cores (mixed) and on the tensor pipe (mixed_tc), and the
    mixed forms' relative L2 errors."""
    import torch
    from zefr_b200 import meshgen
    mesh = meshgen.box_tris(128, seed=2024, jitter=0.15)
    out = {"workload": "triangles_128x128x2_P4_navier_stokes_roe_ldg", "elements": int(mesh.n_elements)}
    R = {}
    for form in ("mixed", "mixed_tc", "fp64"):
        s = triangle_solver(form, mesh)
        for i in range(W):
            s.compute_residual(i % 4)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for i in range(K):
            s.compute_residual(i % 4)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / K
        dof = s.nspts * s.nvars * s.neles
        s.compute_residual(0)
        R[form] = s.get_residual(0)
        prof = kernel_profile(s, K)
        out[form] = {"gdof_s": dof / (ms * 1e-3) / 1e9, "ms_per_residual": ms, "dof": dof,
                     "kernels_ms": {k: v["ms_avg"] for k, v in prof.items() if v["launches"]}}
        if form == "fp64":
            # the triangle adjoint: one (d divF/dU)^T lam against one FP64 residual
            adj = time_adjoint(s, s.get_state(), K, W)
            out["adjoint"] = {"ms_per_vjp": adj["ms_per_vjp"], "kernels": adj["kernels"],
                              "adjoint_over_forward": adj["ms_per_vjp"] / sum(out[form]["kernels_ms"].values())}
        s.close()
    nrm = np.linalg.norm(R["fp64"])
    out["mixed_rel_l2_err_vs_fp64"] = float(np.linalg.norm(R["mixed"] - R["fp64"]) / nrm)
    out["mixed_tc_rel_l2_err_vs_fp64"] = float(np.linalg.norm(R["mixed_tc"] - R["fp64"]) / nrm)
    out["mixed_over_fp64"] = out["fp64"]["ms_per_residual"] / out["mixed"]["ms_per_residual"]
    out["mixed_tc_over_mixed"] = out["mixed"]["ms_per_residual"] / out["mixed_tc"]["ms_per_residual"]
    return out


def batched_side(steps: int = 5, ncases: int = 512, seed: int = 4):
    """Batched vortex workload: 512 independent periodic quad meshes n x n on
    [-5,5]^2 (n uniform in [8,96]), P uniform in 1..5, isentropic vortex of
    strength uniform in [1,5] at a centre uniform in [-2,2]^2 on a stream of
    Mach uniform in [0.2,0.8], all from one seed; mixed form.  Throughput of
    the autotuned persistent stages under a CUDA graph against the same cases
    stepped one launch per case and stage."""
    from zefr_b200 import batch as zbatch
    t0 = time.perf_counter()
    cases = zbatch.vortex_cases(ncases, seed, precision="mixed")
    setup_s = time.perf_counter() - t0
    dof = sum(c.nspts * c.nvars * c.neles for c in cases)
    bt = zbatch.Batch(cases)
    cfg = bt.autotune(steps=2)
    bt.step(2)
    bt.synchronize()
    n0 = bt.launch_count()
    t0 = time.perf_counter()
    bt.step(steps)
    bt.synchronize()
    ms_batch = (time.perf_counter() - t0) * 1e3 / steps
    batch_launches = (bt.launch_count() - n0) // steps
    # the other form at its own best launch shape: one launch per stage for
    # all orders, or one per order, whichever the autotuner did not pick
    cfg_other = bt.autotune(steps=2, form=not cfg["fused"])
    bt.step(2)
    bt.synchronize()
    n1 = bt.launch_count()
    t0 = time.perf_counter()
    bt.step(steps)
    bt.synchronize()
    ms_other = (time.perf_counter() - t0) * 1e3 / steps
    other_launches = (bt.launch_count() - n1) // steps
    # one launch per case and stage, every case on its own context stream
    for c in cases:
        c.step(1)
    for c in cases:
        c.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for c in cases:
            c.step(1)
    for c in cases:
        c.synchronize()
    ms_single = (time.perf_counter() - t0) * 1e3 / steps
    # the same launches serialised on one stream (a host loop over cases)
    import torch
    shared = torch.cuda.Stream()
    for c in cases:
        c.set_stream(shared.cuda_stream)
    for c in cases:
        c.step(1)
    shared.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        for c in cases:
            c.step(1)
    shared.synchronize()
    ms_serial = (time.perf_counter() - t0) * 1e3 / steps
    res_per_step = 4  # RK44 stages, one residual each
    out = {"workload": "batched_vortex_512_quads_n8-96_P1-5_euler", "cases": ncases, "dof": dof,
           "setup_s": setup_s, "autotuned": cfg,
           "batched": {"gdof_s": dof * res_per_step / (ms_batch * 1e-3) / 1e9, "ms_per_step": ms_batch,
                       "launches_per_step": batch_launches,
                       "kernels": ("one persistent kernel per stage for all orders" if cfg["fused"] else
                                   "one persistent kernel per order present and stage, concurrent streams")},
           "one_launch_per_case": {"gdof_s": dof * res_per_step / (ms_single * 1e-3) / 1e9,
                                   "ms_per_step": ms_single, "launches_per_step": 4 * ncases,
                                   "streams": "one per case (concurrent)"},
           "one_launch_per_case_one_stream": {"gdof_s": dof * res_per_step / (ms_serial * 1e-3) / 1e9,
                                              "ms_per_step": ms_serial, "launches_per_step": 4 * ncases},
           "timing": "host clock around synchronised steps (both paths), 4 residuals per RK44 step"}
    out["other_form"] = {"form": "one launch per stage (all orders)" if not cfg["fused"] else
                         "one launch per order and stage", "gdof_s": dof * res_per_step / (ms_other * 1e-3) / 1e9,
                         "ms_per_step": ms_other, "launches_per_step": other_launches, "autotuned": cfg_other}
    out["batched_over_single"] = ms_single / ms_batch
    out["batched_over_single_one_stream"] = ms_serial / ms_batch
    bt.close()
    for c in cases:
        c.close()
    return out


def cylinder_adjoint_side(nsteps: int = 500, every: int = 50):
    """Cylinder adjoint workload: curved O-mesh of 48 x 96 nine-node quads
    (r 0.5 to 20, stretch 1.1), P3, Ma 0.2, Re 100, characteristic far field,
    adiabatic no-slip wall; objective = drag averaged over 500 RK44 steps;
    gradient with respect to 16 wall Fourier coefficients and the free-stream
    angle through the hand-written adjoint, checkpoints every 50 steps, FP64.
    Checked against central differences (step 1e-6, and Richardson's
    extrapolation from steps 1e-6 and 2e-6, which removes the difference's own
    h^2 error) of the forward run for the first, the third (the largest
    component) and the last wall coefficient and the angle."""
    from zefr_b200.shape import CylinderDrag
    prob = CylinderDrag(nr=48, nt=96, order=3, dt=1e-4, checkpoint_every=every)
    coef = np.zeros(16)
    coef[:4] = (0.01, -0.005, 0.003, 0.002)
    alpha = 0.05
    prob.drag(coef, alpha, 2)  # warm-ups of both paths (library, torch.func and allocator set-up)
    prob.gradient(coef, alpha, 2)
    # best of three runs of each: the host-side share (one library call per
    # step, the objective's torch evaluation per checkpoint segment) varies
    # from run to run
    t_fwd = t_adj = float("inf")
    for _ in range(3):
        t0 = time.perf_counter()
        J = prob.drag(coef, alpha, nsteps)
        t_fwd = min(t_fwd, time.perf_counter() - t0)
        t0 = time.perf_counter()
        g = prob.gradient(coef, alpha, nsteps)
        t_adj = min(t_adj, time.perf_counter() - t0)
    h = 1e-6
    gmax = max(float(np.abs(g["dJ_dcoef"]).max()), abs(g["dJ_dalpha"]))

    def fd(k, step):
        """central difference in coefficient k (k = -1: the angle)"""
        if k < 0:
            return (prob.drag(coef, alpha + step, nsteps) - prob.drag(coef, alpha - step, nsteps)) / (2 * step)
        cp, cm = coef.copy(), coef.copy()
        cp[k] += step
        cm[k] -= step
        return (prob.drag(cp, alpha, nsteps) - prob.drag(cm, alpha, nsteps)) / (2 * step)

    checks = {}
    for k in (0, 2, 15, -1):
        adj = float(g["dJ_dcoef"][k]) if k >= 0 else float(g["dJ_dalpha"])
        d1, d2 = fd(k, h), fd(k, 2 * h)
        rich = (4.0 * d1 - d2) / 3.0  # Richardson: removes the h^2 term of the central difference
        checks["alpha" if k < 0 else f"coef{k}"] = {
            "adjoint": adj, "central_difference": d1, "central_difference_richardson": rich,
            "rel_err": abs(adj - d1) / abs(d1), "rel_err_richardson": abs(adj - rich) / abs(rich),
            "err_over_largest_gradient_component": abs(adj - d1) / gmax}
    return {"workload": "cylinder_omesh_48x96_quad9_P3_ns_drag_adjoint", "steps": nsteps,
            "checkpoint_every": every, "J_mean_drag": J,
            "dJ_dcoef": [float(x) for x in g["dJ_dcoef"]], "dJ_dalpha": g["dJ_dalpha"],
            "fd_check": checks,
            "forward_s": t_fwd, "gradient_s": t_adj, "gradient_over_forward": t_adj / t_fwd,
            "timing": "host clock, best of three runs each, both including their mesh set-up; the gradient run "
                      "includes its own forward pass, the checkpoint recomputation and 500 RK44 step adjoints "
                      "(2,000 stage adjoints)"}


def cpu_baseline_sample(steps: int = 8, warmup: int = 1):
    """Reference CPU residual on a bounded sample: this script's reference arm
    (the compiled reference, release flags, OpenMP on all host cores, TGV
    REF_CELLS^3 with Rusanov) run as a subprocess, so no thread of this
    process (torch, CUDA) competes with its OpenMP team; both CPU figures in
    a run then come from the same code on the same sample."""
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    env["OMP_NUM_THREADS"] = str(os.cpu_count() or 1)
    try:
        out = subprocess.run([sys.executable, os.path.abspath(__file__), "--impl", "reference", "--steps", str(steps),
                              "--warmup", str(warmup)], env=env, capture_output=True, text=True, timeout=600)
    except (subprocess.TimeoutExpired, OSError) as e:
        return {"unavailable": f"reference CPU sample failed: {e}"}
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    if out.returncode != 0 or not lines:
        return {"unavailable": "reference CPU sample failed: " + (out.stderr.strip().splitlines() or ["?"])[-1]}
    ref = json.loads(lines[-1])
    if "unavailable" in ref:
        return {"unavailable": ref["unavailable"]}
    cb = dict(ref["cpu_baseline"])
    cb["ms_per_residual"] = ref["ms_per_step"]
    return cb


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def mixed_errors(n: int, U: np.ndarray, R64: np.ndarray, steps: int = 60, every: int = 10):
    """Errors of the mixed form against the FP64 form on the bench workload:
    residual on the same FP64 input (the gate), residual on the state the
    mixed form actually stores (both forms fed the FP32-rounded state: the
    arithmetic's share), the state after ``steps`` RK44 steps (relative to the
    state and to its change), and the kinetic-energy and dissipation-rate
    histories sampled every ``every`` steps."""
    import torch
    out = {}
    sm, _ = build_solver("mixed", n)
    s64, _ = build_solver("fp64", n)
    sm.set_state(U)
    sm.compute_residual(0)
    Rm = sm.get_residual(0)
    nrm = np.linalg.norm(R64)
    out["residual_rel_l2"] = float(np.linalg.norm(Rm - R64) / nrm)
    var_err = [float(np.linalg.norm(Rm[:, v] - R64[:, v]) / np.linalg.norm(R64[:, v])) for v in range(U.shape[1])]
    out["residual_rel_l2_per_variable"] = var_err
    # both forms on the state the mixed form stores
    Uq = sm.get_state()
    s64.set_state(Uq)
    s64.compute_residual(0)
    R64q = s64.get_residual(0)
    sm.set_state(Uq)
    sm.compute_residual(0)
    Rmq = sm.get_residual(0)
    out["residual_rel_l2_same_stored_state"] = float(np.linalg.norm(Rmq - R64q) / np.linalg.norm(R64q))
    out["residual_rel_l2_fp64_rounded_vs_exact_input"] = float(np.linalg.norm(R64q - R64) / nrm)
    # trajectories
    hist = {}
    states = {}
    for name, s in (("mixed", sm), ("fp64", s64)):
        s.set_state(U)
        ke = []
        for _ in range(steps // every):
            ke.append(s.functionals()["ke"])
            s.step(every)
        ke.append(s.functionals()["ke"])
        hist[name] = np.array(ke)
        states[name] = s.get_state()
    d = states["mixed"] - states["fp64"]
    out["state_rel_l2_after_steps"] = float(np.linalg.norm(d) / np.linalg.norm(states["fp64"]))
    out["state_rel_l2_of_change_after_steps"] = float(np.linalg.norm(d) / np.linalg.norm(states["fp64"] - U))
    ke64, kem = hist["fp64"], hist["mixed"]
    out["ke_history_rel_err"] = float(np.abs(kem - ke64).max() / np.abs(ke64).max())
    eps64, epsm = -np.diff(ke64), -np.diff(kem)
    out["dissipation_rel_err"] = float(np.abs(epsm - eps64).max() / np.abs(eps64).max())
    out["steps"] = steps
    out["dt"] = TGV_DECK["dt"]
    sm.close()
    s64.close()
    torch.cuda.empty_cache()
    return out


def timed_form(form: str, n: int, K: int, W: int, world: int, local: int, U=None, flux: str = "roe",
               extras: bool = True):
    """CUDA-event time per residual of one form (max over ranks), with the
    clocks sampled during the timed region, the per-kernel split, the RK stage
    time and, with ``extras``, the residual at the input state (rank 0), the
    FP64 adjoint and the end-to-end time through host buffers."""
    import torch
    s, U_form = build_solver(form, n, flux)
    U = U_form if U is None else U
    s.set_state(U)
    clocks = Clocks(local)
    clocks.start()
    ms, nl = time_residuals(s, K, W, world)
    clk = clocks.stop()
    out = {"ms": ms, "launches": nl, "clocks": clk, "prof": kernel_profile(s, K)}
    geom = (s.nspts, s.nvars, s.neles, s.ndims, s.info.nfpts, int(s.info.n_gfpts))
    if extras:
        out["rk"] = time_rk_stage(s, K, world)
        out["adj"] = time_adjoint(s, U, K, W) if form == "fp64" else None
        rank = dist_env()[0]
        s.set_state(U)
        s.compute_residual(0)
        out["R"] = s.get_residual(0) if rank == 0 else None
        out["e2e"] = time_e2e(s, U, max(3, min(K, 10)), min(W, 2), world)
    s.close()
    del s
    torch.cuda.empty_cache()
    return out, U, geom


def gpu_arm(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    else:
        torch.cuda.set_device(0)
    n = args.cells
    K, W = args.steps, args.warmup
    f64, U, geom = timed_form("fp64", n, K, W, world, local)
    mixed, _, _ = timed_form("mixed", n, K, W, world, local, U=U)
    rus, _, _ = timed_form("fp64", n, K, W, world, local, U=U, flux="rusanov", extras=False)
    errs = mixed_errors(n, U, f64["R"]) if rank == 0 else None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    S, V, E, D, Fp, G = geom
    dof = S * V * E
    gate_met = errs["residual_rel_l2"] <= MIXED_GATE
    head, head_name = (mixed, "mixed") if gate_met else (f64, "fp64")
    w = 4 if gate_met else 8
    peak, peak_kind = measured_peaks()
    res_kernels = [k for k in head["prof"] if k in ("k_extrap", "k_ns_grad", "k_ns_face", "k_euler")]
    t_res = sum(head["prof"][k]["ms_avg"] for k in res_kernels)
    dom = max(res_kernels, key=lambda k: head["prof"][k]["ms_avg"])
    bytes_alg = b_alg(E, S, V, D, G, Fp, w)
    achieved = bytes_alg / (t_res * 1e-3) / 1e9
    traffic = (MIXED_DRAM_BYTES_PER_ELEMENT if gate_met else FP64_DRAM_BYTES_PER_ELEMENT) * E
    t_res64 = sum(f64["prof"][k]["ms_avg"] for k in f64["prof"] if k in res_kernels)
    t_resm = sum(mixed["prof"][k]["ms_avg"] for k in mixed["prof"] if k in res_kernels)
    e2e_ms, h2d, d2h = head["e2e"]
    gd = lambda ms: world * dof / (ms * 1e-3) / 1e9  # noqa: E731
    line = {
        "metric": METRIC,
        "value": gd(head["ms"]),
        "unit": "GDOF/s",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": head["ms"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if gate_met else "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "mesh": f"{n}^3 linear hexes, periodic [0,2pi]^3", "order": ORDER,
                   "dof_per_gpu": dof, "elements_per_gpu": E, "flux": "Roe + LDG (beta 0.5, tau 0.1)",
                   "Re": 1600, "Ma": 0.1, "step": "one compute_residual(stage) incl. extrapolation",
                   "form": head_name,
                   "l2": "inputs larger than L2 (mixed state 336 MB, FP64 state 671 MB)",
                   "parallelism": "replicas only" if world > 1 else "single GPU"},
        "headline_form": head_name,
        "mixed_gate": {"quantity": "relative L2 error of the mixed residual against the FP64 residual on the same "
                                   "input state", "bound": MIXED_GATE, "value": errs["residual_rel_l2"],
                       "met": gate_met},
        "fp64": {"value": gd(f64["ms"]), "ms_per_step": f64["ms"], "dtype": "f64", "rk_stage_ms": f64["rk"],
                 "kernels": f64["prof"], "kernel_ms_per_residual": t_res64,
                 "roofline_frac_of_measured": b_alg(E, S, V, D, G, Fp, 8) / (t_res64 * 1e-3) / 1e9 / peak},
        "mixed": {"value": gd(mixed["ms"]), "ms_per_step": mixed["ms"], "dtype": "f32", "rk_stage_ms": mixed["rk"],
                  "kernels": mixed["prof"], "kernel_ms_per_residual": t_resm,
                  "roofline_frac_of_measured": b_alg(E, S, V, D, G, Fp, 4) / (t_resm * 1e-3) / 1e9 / peak,
                  "errors_vs_fp64": errs,
                  "form": "FP32 state (deviation from its mean), traces, metrics, residual and arithmetic "
                          "(inviscid flux as deviation from the reference state); FP64 set-up and reductions; "
                          "Kahan-compensated RK44",
                  "e2e_gdof_s": gd(mixed["e2e"][0])},
        "mixed_over_fp64": f64["ms"] / mixed["ms"],
        "fp64_rusanov": {"value": gd(rus["ms"]), "ms_per_step": rus["ms"], "kernels": rus["prof"],
                         "note": "same workload with the Rusanov common flux, the reference's only inviscid flux"},
        "adjoint": {"form": "FP64", "ms_per_vjp": f64["adj"]["ms_per_vjp"], "forward_residual_ms": t_res64,
                    "adjoint_over_forward": f64["adj"]["ms_per_vjp"] / t_res64,
                    "kernels": f64["adj"]["kernels"],
                    "note": "kernel time of one (d divF/dU)^T lam at the TGV state vs one FP64 residual "
                            "(the same kernels' CUDA-event times)"},
        "rk_stage_ms": head["rk"],
        "kernels": head["prof"],
        "gpu_launches": head["launches"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": f"{head_name} residual = " + " + ".join(res_kernels) + f" (dominant {dom})",
                     "algorithmic_bytes_per_launch": bytes_alg, "peak_kind": peak_kind},
        "e2e": {"value": gd(e2e_ms), "unit": "GDOF/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "path": f"{head_name} form: zb_compute_residuals_host over the timed steps (per step: pinned "
                        "host state to device, zb_compute_residual, residual to pinned host; copies of "
                        "neighbouring steps overlap the residual)"},
        "clocks": head["clocks"],
    }
    if world == 1 and not args.no_cpu:
        cb = cpu_baseline_sample()
        if "unavailable" not in cb:
            cb["cpu_model"] = cpu_model()
        line["cpu_baseline"] = cb
    if world == 1 and not args.no_side:
        torch.cuda.empty_cache()
        line["triangles"] = triangle_side(K, W)
        torch.cuda.empty_cache()
        line["batched"] = batched_side()
        torch.cuda.empty_cache()
        line["cylinder_adjoint"] = cylinder_adjoint_side()
    return line


def profile_run(args):
    """Short run of one form for an external profiler: W + K residuals (or
    adjoint applications at the FP64 form, or, for "opmm", tensor-core
    products of the hexahedral P3 extrapolation operator's shape, 96 x 64, on
    5 n^3 columns), no timing."""
    import torch
    torch.cuda.set_device(0)
    if args.profile_form == "opmm":
        from zefr_b200 import _lib
        fp = ctypes.POINTER(ctypes.c_float)
        m, k, n = 96, 64, 5 * args.cells ** 3
        g = torch.Generator(device="cuda").manual_seed(1)
        A = torch.randn(m, k, device="cuda", generator=g)
        B = torch.randn(k, n, device="cuda", generator=g)
        C = torch.empty(m, n, device="cuda")
        for _ in range(args.warmup + args.steps):
            st = _lib.lib().zb_operator_mm_tf32x3(m, n, k, 1.0, ctypes.cast(A.data_ptr(), fp), k,
                                                  ctypes.cast(B.data_ptr(), fp), n, 0.0,
                                                  ctypes.cast(C.data_ptr(), fp), n, None)
            if st != 0:
                raise RuntimeError(_lib.lib().zb_last_error().decode())
        torch.cuda.synchronize()
        return
    adj = args.profile_form == "adjoint"
    if args.profile_form.startswith("tri-"):
        s = triangle_solver(args.profile_form[4:])
    else:
        s, U = build_solver("fp64" if adj else args.profile_form, args.cells)
        s.set_state(U)
    lam = torch.ones(s.state_shape, dtype=torch.float64, device="cuda") if adj else None
    for i in range(args.warmup + args.steps):
        if adj:
            s.vjp(lam)
        else:
            s.compute_residual(i % 4)
    torch.cuda.synchronize()
    s.close()


# ---------------------------------------------------------------------------
# reference arm (CPU)
# ---------------------------------------------------------------------------

def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return None
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if world > 1:
        # torchrun sets OMP_NUM_THREADS=1 for every rank; only this rank works
        # here, so the reference gets all host cores (the environment for an
        # OpenMP runtime not loaded yet, the call for one already loaded)
        threads = os.cpu_count() or 1
        os.environ["OMP_NUM_THREADS"] = str(threads)
        try:
            ctypes.CDLL("libgomp.so.1").omp_set_num_threads(threads)
        except (OSError, AttributeError):
            pass
    from oracle import refcpu
    if not refcpu.available(fast=True):
        return {"impl": "reference", "unavailable": "oracle/_ref/libzefr_ref_fast.so not built (make -C oracle)"}
    from zefr_b200 import ics, meshgen
    n = args.ref_cells
    with tempfile.TemporaryDirectory() as tmp:
        mesh = meshgen.box_hexes(n, n, n)
        meshgen.write_gmsh(mesh, os.path.join(tmp, "tgv.msh"))
        deck = {k: v for k, v in TGV_DECK.items() if k not in ("ndims", "order", "viscous")}
        refcpu.write_deck(os.path.join(tmp, "tgv.deck"), "tgv.msh", 3, ORDER, True, {"PERIODIC": "periodic"}, deck)
        r = refcpu.RefSolver(os.path.join(tmp, "tgv.deck"), fast=True)
        S, V, E = r.state_shape
        X = r.array("coord_spts").reshape(S, 3, E)
        r.set_state(ics.taylor_green(X, mach=TGV_DECK["mach_fs"]))
        for i in range(args.warmup):
            r.compute_residual(i % 4)
        t0 = time.perf_counter()
        for i in range(args.steps):
            r.compute_residual(i % 4)
        dt = (time.perf_counter() - t0) / args.steps
        r.close()
    dof = S * V * E
    value = dof / dt / 1e9
    sample = (f"reference CPU FRSolver::compute_residual (-Ofast, OpenMP {threads} threads, GiMMiK stand-in GEMM; "
              f"compute_F serial in the reference) on TGV {n}^3 hex P3 NS with Rusanov + LDG ({dof} DOF), "
              f"one residual per step; the reference has no Roe flux")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"taylor_green_{n}^3_hex_P3_navier_stokes_rusanov_ldg",
                       "sample_of": WORKLOAD, "mesh": f"{n}^3 linear hexes, periodic [0,2pi]^3", "order": ORDER,
                       "dof": dof, "flux": "Rusanov + LDG (beta 0.5, tau 0.1)", "Re": 1600, "Ma": 0.1,
                       "cores": threads, "cpu_model": cpu_model()},
            "cpu_baseline": {"value": value, "unit": "GDOF/s", "cores": threads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=NCELL, help=argparse.SUPPRESS)
    ap.add_argument("--ref-cells", type=int, default=REF_CELLS, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--no-side", action="store_true", help="skip the triangle and batched side workloads")
    ap.add_argument("--profile-form", choices=["mixed", "fp64", "adjoint", "tri-mixed", "tri-mixed_tc", "tri-fp64",
                                               "opmm"],
                    default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_form:
        profile_run(args)
        return
    line = reference_arm(args) if args.impl == "reference" else gpu_arm(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
