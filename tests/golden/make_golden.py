"""Generate the golden fixtures in tests/golden/*.npz from the reference solver.

Runs the reference's own CPU FRSolver (built by ``make -C oracle``) on small
synthetic meshes of every workload shape, with seeded states, and stores:

  mesh          nodes, elements, boundary faces, boundary-condition map
  params        the reference InputStruct values after its non-dimensionalisation
  setup arrays  the reference's operators, metrics and per-flux-point face data
  U0, R0        input state and divF_spts(0) = reference compute_residual(0)
  Un            state after ``nsteps`` reference RK44 steps (FRSolver::update)

under tests/golden/diag/, the reference's own diagnostics at U0 after
compute_residual(0) (report_residuals for res_type 0/1/2, report_turbulent_stats
for 3D Navier-Stokes, compute_moments for cases with walls), under
tests/golden/traj/ long RK44 trajectories (the state after every block of
steps), and, under tests/golden/time/, time-integration cases (RK54 with and without
the adaptive controller, RK44 with CFL time steps) holding the mesh, deck,
U0, the reference's dt(0) after every step, its per-element dt array after
the last step and the final state.

Usage:  python tests/golden/make_golden.py [names]  (needs oracle/_ref/libzefr_ref.so)
"""
from __future__ import annotations

import json
import math
import os
import sys
import tempfile
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refcpu  # noqa: E402
from zefr_b200 import ics, meshgen  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))

# name -> (mesh builder, ndims, order, viscous, bounds, deck params, state builder, nsteps)
def _cases():
    tgv_deck = {"disable_nondim": 1, "fix_vis": 1, "mach_fs": 0.1, "Re_fs": 1600, "prandtl": 0.71,
                "P_fs": 1.0, "rho_fs": 1.0, "L_fs": 1.0, "ldg_b": 0.5, "ldg_tau": 0.1, "dt": 1e-3}
    cyl_deck = {"disable_nondim": 1, "fix_vis": 1, "mach_fs": 0.2, "Re_fs": 100, "prandtl": 0.72,
                "P_fs": 1.0, "rho_fs": 1.0, "L_fs": 1.0, "ldg_b": 0.5, "ldg_tau": 0.1, "dt": 1e-3}
    eul = {"mach_fs": 0.3, "rho_fs": 1.0, "P_fs": 1.0, "dt": 1e-3}

    def vortex(X, g):
        return ics.isentropic_vortex(X, beta=5.0, gamma=g)

    def tgv(X, g):
        return ics.taylor_green(X, mach=0.1, gamma=g)

    def tgv_fast(X, g):
        return ics.taylor_green(X, mach=0.3, gamma=g)

    def cyl_state(X, g):
        c = 0.2 * np.sqrt(g)
        return ics.uniform(X, 1.0, (c, 0.0), 1.0, g)

    def shear(X, g):
        return ics.double_shear_layer(X * 0.1 + 0.5, mach=0.2, gamma=g)

    def angled_state(X, g):
        c = 0.2 * np.sqrt(g)
        return ics.uniform(X, 1.0, (c * math.cos(math.pi / 6), c * math.sin(math.pi / 6)), 1.0, g)

    def shear_unit(X, g):
        return ics.double_shear_layer(X, mach=0.2, gamma=g)

    per = {"PERIODIC": "periodic"}
    return {
        "quad_p3_euler_vortex": (lambda: meshgen.box_quads(8, 8), 2, 3, False, per, eul, vortex, 3),
        "quad_p2_ns_jitter": (lambda: meshgen.jitter_interior(meshgen.box_quads(6, 5), 0.4, 11), 2, 2, True, per,
                              dict(cyl_deck, ldg_tau=1.0), shear, 2),
        "quad_p1_euler": (lambda: meshgen.box_quads(5, 5), 2, 1, False, per, eul, vortex, 2),
        "quad_p5_euler": (lambda: meshgen.box_quads(4, 4), 2, 5, False, per, eul, vortex, 2),
        "hex_p3_ns_tgv": (lambda: meshgen.box_hexes(3, 3, 3), 3, 3, True, per, tgv_deck, tgv, 2),
        "hex_p2_euler_jitter": (lambda: meshgen.jitter_interior(meshgen.box_hexes(3, 4, 2), 0.15, 5), 3, 2, False,
                                per, eul, tgv_fast, 2),
        "hex_p1_ns": (lambda: meshgen.box_hexes(3, 2, 2), 3, 1, True, per, tgv_deck, tgv, 2),
        "hex_p4_euler": (lambda: meshgen.box_hexes(2, 2, 2), 3, 4, False, per, eul, tgv_fast, 1),
        "cyl_p3_ns_char_adi": (lambda: meshgen.cylinder_omesh(4, 8, r1=5.0), 2, 3, True,
                               {"WALL": "wall_ns_adi", "FARFIELD": "char"}, cyl_deck, cyl_state, 2),
        "cyl_p2_ns_iso_farfield_b03": (lambda: meshgen.cylinder_omesh(3, 8, r1=4.0), 2, 2, True,
                                       {"WALL": "wall_ns_iso", "FARFIELD": "farfield"},
                                       {"mach_fs": 0.2, "Re_fs": 100, "fix_vis": 0, "ldg_b": 0.3, "ldg_tau": 0.2,
                                        "T_wall": 300.0, "dt": 1e-4}, None, 2),
        "cyl_p3_euler_slip_char": (lambda: meshgen.cylinder_omesh(4, 8, r1=5.0), 2, 3, False,
                                   {"WALL": "wall_slip", "FARFIELD": "char"}, dict(eul, mach_fs=0.2), cyl_state, 2),
        "cyl_p2_euler_supin_sym": (lambda: meshgen.cylinder_omesh(3, 8, r1=4.0), 2, 2, False,
                                   {"WALL": "symmetry", "FARFIELD": "farfield"}, dict(eul, mach_fs=0.2), cyl_state, 2),
        # triangles (FR with Williams-Shunn points and the 'M3' correction)
        "tri_p4_ns_jitter": (lambda: meshgen.box_tris(4, seed=3), 2, 4, True, per,
                             dict(cyl_deck, Re_fs=1000, prandtl=0.71), shear_unit, 2),
        "tri_p2_euler_vortex": (lambda: meshgen.box_tris(5, -5.0, 5.0, seed=1), 2, 2, False, per, eul, vortex, 2),
        # free stream at 30 degrees: no boundary of the box is tangent to the
        # flow, where the characteristic condition's inflow/outflow switch
        # would follow the rounding of the normal
        "tri_p3_euler_char": (lambda: meshgen.box_tris(4, -2.0, 2.0, seed=2, bnd="FARFIELD"), 2, 3, False,
                              {"FARFIELD": "char"},
                              dict(eul, mach_fs=0.2, nx_fs=math.cos(math.pi / 6), ny_fs=math.sin(math.pi / 6)),
                              angled_state, 2),
        "tri_p1_ns_adi": (lambda: meshgen.box_tris(4, 0.0, 1.0, seed=4, bnd="WALL"), 2, 1, True,
                          {"WALL": "wall_ns_adi"}, cyl_deck, shear_unit, 2),
        # higher orders (Williams-Shunn points P5-P8)
        "tri_p5_ns_jitter": (lambda: meshgen.box_tris(3, seed=5), 2, 5, True, per,
                             dict(cyl_deck, Re_fs=1000, prandtl=0.71), shear_unit, 2),
        "tri_p6_euler_vortex": (lambda: meshgen.box_tris(3, -5.0, 5.0, seed=6), 2, 6, False, per, eul, vortex, 2),
        "tri_p7_ns_adi": (lambda: meshgen.box_tris(3, 0.0, 1.0, seed=7, bnd="WALL"), 2, 7, True,
                          {"WALL": "wall_ns_adi"}, cyl_deck, shear_unit, 1),
        "tri_p8_euler_char": (lambda: meshgen.box_tris(2, -2.0, 2.0, seed=8, bnd="FARFIELD"), 2, 8, False,
                              {"FARFIELD": "char"},
                              dict(eul, mach_fs=0.2, nx_fs=math.cos(math.pi / 6), ny_fs=math.sin(math.pi / 6)),
                              angled_state, 1),
    }


def reference_setup(r: refcpu.RefSolver):
    """Reference set-up arrays in the per-element-flux-point form of oracle.dfr_numpy.Setup."""
    Fp, E, D = r.nfpts, r.neles, r.ndims
    g = r.array("fpt2gfpt").astype(np.int64).reshape(Fp, E)
    sl = r.array("fpt2gfpt_slot").astype(np.int64).reshape(Fp, E)
    nG = r.ngfpts
    gfpt2bnd = r.array("gfpt2bnd").astype(np.int64)
    owners = np.full((nG, 2), -1, dtype=np.int64)
    for e in range(E):
        for f in range(Fp):
            owners[g[f, e], sl[f, e]] = e * Fp + f
    partner = np.empty((Fp, E), dtype=np.int64)
    for e in range(E):
        for f in range(Fp):
            gg = g[f, e]
            if gg < r.ngfpts_int:
                partner[f, e] = owners[gg, 1 - sl[f, e]]
            else:
                partner[f, e] = -1 - gfpt2bnd[gg - r.ngfpts_int]
    norm = r.array("norm").reshape(D, nG)
    dA = r.array("dA").reshape(2, nG)
    fnorm = np.transpose(norm[:, g], (1, 0, 2))            # [Fp, D, E]
    fdA = np.take_along_axis(dA[:, g.reshape(-1)], sl.reshape(1, -1), axis=0).reshape(Fp, E)
    S = r.nspts
    return {
        "oppE": r.array("oppE"), "oppD": r.array("oppD"), "oppD_fpts": r.array("oppD_fpts"),
        "oppDiv": r.array("oppDiv"), "oppDiv_fpts": r.array("oppDiv_fpts"),
        "inv_jaco_spts": r.array("inv_jaco_spts"), "jaco_det_spts": r.array("jaco_det_spts"),
        "coord_spts": r.array("coord_spts"),
        "fpt_partner": partner.reshape(-1).astype(np.float64), "fpt_slot": sl.reshape(-1).astype(np.float64),
        "fpt_norm": fnorm.reshape(-1), "fpt_dA": fdA.reshape(-1),
    }


def make_case(name, spec, tmp):
    build, ndims, order, viscous, bounds, deck, state_fn, nsteps = spec
    mesh = build()
    msh = os.path.join(tmp, name + ".msh")
    meshgen.write_gmsh(mesh, msh)
    deck_path = refcpu.write_deck(os.path.join(tmp, name + ".deck"), name + ".msh", ndims, order, viscous,
                                  bounds, deck)
    r = refcpu.RefSolver(deck_path)
    S, V, E = r.state_shape
    X = r.array("coord_spts").reshape(S, ndims, E)
    g = r.params["gamma"]
    if state_fn is None:  # free stream at the reference's non-dimensional values
        p = r.params
        U0 = ics.uniform(X, p["rho_fs"], (p["V_fs0"], p["V_fs1"], p["V_fs2"]), p["P_fs"], g)
    else:
        U0 = state_fn(X, g)
    # Triangles: 5% perturbations, so residuals are not a 1e-3 difference of
    # O(1) fluxes; their dense operators come out of a Vandermonde inverse
    # that agrees with the reference's (Eigen LU) only to rounding.
    amp = 5e-2 if name.startswith("tri_") else 1e-3
    U0 = ics.perturb(U0, amp, seed=zlib.crc32(name.encode()))
    R0 = r.residual(U0, 0)
    r.set_state(U0)
    r.update(nsteps)
    Un = r.get_state()
    setup = reference_setup(r)
    faces_t = np.array([f[0] for f in mesh.bnd_faces], dtype=np.int64)
    npf = max(len(f[1]) for f in mesh.bnd_faces)
    faces_n = np.full((len(mesh.bnd_faces), npf), -1, dtype=np.int64)
    for i, f in enumerate(mesh.bnd_faces):
        faces_n[i, :len(f[1])] = f[1]
    faces_name = np.array([f[2] for f in mesh.bnd_faces])
    meta = {"name": name, "ndims": ndims, "order": order, "viscous": bool(viscous), "bounds": bounds,
            "deck": deck, "params": r.params, "nsteps": nsteps, "dt": r.params["dt"],
            "shape": [S, V, E], "nfpts": r.nfpts, "gmsh_type": mesh.gmsh_type}
    out = os.path.join(HERE, name + ".npz")
    np.savez_compressed(out, meta=json.dumps(meta), nodes=mesh.nodes, elements=mesh.elements, faces_type=faces_t,
                        faces_nodes=faces_n, faces_name=faces_name, U0=U0, R0=R0, Un=Un,
                        **{"setup_" + k: v for k, v in setup.items()})
    r.close()
    return out


# name -> (mesh builder, ndims, order, viscous, bounds, deck params incl. time keys, state builder, nsteps)
def _time_cases():
    cyl_deck = {"disable_nondim": 1, "fix_vis": 1, "mach_fs": 0.2, "Re_fs": 100, "prandtl": 0.72,
                "P_fs": 1.0, "rho_fs": 1.0, "L_fs": 1.0, "ldg_b": 0.5, "ldg_tau": 0.1}
    eul = {"mach_fs": 0.3, "rho_fs": 1.0, "P_fs": 1.0}

    def vortex(X, g):
        return ics.isentropic_vortex(X, beta=5.0, gamma=g)

    def shear(X, g):
        return ics.double_shear_layer(X * 0.1 + 0.5, mach=0.2, gamma=g)

    def tgv(X, g):
        return ics.taylor_green(X, mach=0.3, gamma=g)

    def cyl_state(X, g):
        c = 0.2 * np.sqrt(g)
        return ics.uniform(X, 1.0, (c, 0.0), 1.0, g)

    per = {"PERIODIC": "periodic"}
    quads = lambda: meshgen.box_quads(6, 6)  # noqa: E731
    jq = lambda: meshgen.jitter_interior(meshgen.box_quads(6, 5), 0.4, 11)  # noqa: E731
    jh = lambda: meshgen.jitter_interior(meshgen.box_hexes(3, 3, 2), 0.15, 5)  # noqa: E731
    return {
        "rk54_quad_p3_vortex": (quads, 2, 3, False, per, dict(eul, dt=5e-3, dt_scheme="RK54"), vortex, 3),
        # the first step is rejected (dt 0.2 is far too large) and redone
        "rk54_adapt_quad_p3_vortex": (quads, 2, 3, False, per, dict(eul, dt=0.2, dt_scheme="RK54", adapt_dt=1),
                                      vortex, 4),
        "rk54_adapt_hex_p1_ns": (lambda: meshgen.box_hexes(3, 2, 2), 3, 1, True, per,
                                 dict(cyl_deck, mach_fs=0.3, dt=1e-2, dt_scheme="RK54", adapt_dt=1,
                                      err_atol=1e-6, err_rtol=1e-6), tgv, 3),
        "cfl1_global_quad_p2_ns": (jq, 2, 2, True, per,
                                   dict(cyl_deck, ldg_tau=1.0, dt=1e-3, dt_type=1, CFL=0.5, CFL_type=1), shear, 2),
        "cfl2_local_quad_p2_ns": (jq, 2, 2, True, per,
                                  dict(cyl_deck, ldg_tau=1.0, dt=1e-3, dt_type=2, CFL=0.5, CFL_type=2), shear, 2),
        "cfl2_global_hex_p2_ns": (jh, 3, 2, True, per,
                                  dict(cyl_deck, mach_fs=0.3, dt=1e-3, dt_type=1, CFL=0.5, CFL_type=2), tgv, 2),
        "cfl1_local_hex_p2_euler": (jh, 3, 2, False, per, dict(eul, dt=1e-3, dt_type=2, CFL=0.8, CFL_type=1),
                                    tgv, 2),
        "cfl2_global_cyl_p2_ns_char_adi": (lambda: meshgen.cylinder_omesh(3, 8, r1=4.0), 2, 2, True,
                                           {"WALL": "wall_ns_adi", "FARFIELD": "char"},
                                           dict(cyl_deck, dt=1e-4, dt_type=1, CFL=0.5, CFL_type=2), cyl_state, 2),
    }


TIME_DIR = os.path.join(HERE, "time")


def make_time_case(name, spec, tmp):
    build, ndims, order, viscous, bounds, deck, state_fn, nsteps = spec
    mesh = build()
    meshgen.write_gmsh(mesh, os.path.join(tmp, name + ".msh"))
    deck_path = refcpu.write_deck(os.path.join(tmp, name + ".deck"), name + ".msh", ndims, order, viscous,
                                  bounds, deck)
    r = refcpu.RefSolver(deck_path)
    S, V, E = r.state_shape
    X = r.array("coord_spts").reshape(S, ndims, E)
    U0 = ics.perturb(state_fn(X, r.params["gamma"]), 1e-3, seed=zlib.crc32(name.encode()))
    r.set_state(U0)
    dt0 = []
    for _ in range(nsteps):
        r.update(1)
        dt0.append(float(r.array("dt")[0]))
    Un = r.get_state()
    dt_ele = r.array("dt")
    faces_t = np.array([f[0] for f in mesh.bnd_faces], dtype=np.int64)
    npf = max(len(f[1]) for f in mesh.bnd_faces)
    faces_n = np.full((len(mesh.bnd_faces), npf), -1, dtype=np.int64)
    for i, f in enumerate(mesh.bnd_faces):
        faces_n[i, :len(f[1])] = f[1]
    faces_name = np.array([f[2] for f in mesh.bnd_faces])
    meta = {"name": name, "ndims": ndims, "order": order, "viscous": bool(viscous), "bounds": bounds,
            "deck": deck, "params": r.params, "nsteps": nsteps, "shape": [S, V, E], "gmsh_type": mesh.gmsh_type}
    os.makedirs(TIME_DIR, exist_ok=True)
    out = os.path.join(TIME_DIR, name + ".npz")
    np.savez_compressed(out, meta=json.dumps(meta), nodes=mesh.nodes, elements=mesh.elements, faces_type=faces_t,
                        faces_nodes=faces_n, faces_name=faces_name, U0=U0, Un=Un, dt0=np.array(dt0),
                        dt_ele=dt_ele)
    r.close()
    return out


DIAG_DIR = os.path.join(HERE, "diag")
WALL_NAMES = ("wall_slip", "wall_ns_iso", "wall_ns_adi")


def make_diag_case(name, spec, tmp):
    """The reference's diagnostics on the committed golden state U0 of case
    ``name`` (its residual at U0 must equal the committed R0 bit for bit)."""
    build, ndims, order, viscous, bounds, deck, _state_fn, _nsteps = spec
    gold = np.load(os.path.join(HERE, name + ".npz"))
    mesh = build()
    meshgen.write_gmsh(mesh, os.path.join(tmp, name + ".msh"))
    deck_path = refcpu.write_deck(os.path.join(tmp, name + ".deck"), name + ".msh", ndims, order, viscous,
                                  bounds, deck)
    r = refcpu.RefSolver(deck_path)
    R0 = r.residual(gold["U0"], 0)
    if not np.array_equal(R0, gold["R0"]):
        raise RuntimeError(f"{name}: reference residual differs from the committed golden")
    out = {"U0_crc": np.array(zlib.crc32(gold["U0"].tobytes()))}
    for t, key in ((0, "res_max"), (1, "res_l1"), (2, "res_l2")):
        out[key] = r.report_residuals(t)
    if ndims == 3 and viscous:
        ts = r.turbulent_stats()
        out["turb"] = np.array([ts["ke"], ts["enstrophy"], ts["norm"]])
    if any(b in WALL_NAMES for b in bounds.values()):
        m = r.compute_moments()
        out["force"], out["moment"] = m["force"], m["moment"]
    r.close()
    os.makedirs(DIAG_DIR, exist_ok=True)
    path = os.path.join(DIAG_DIR, name + ".npz")
    np.savez_compressed(path, **out)
    return path


TRAJ_DIR = os.path.join(HERE, "traj")


def _traj_cases():
    """name -> (mesh builder, ndims, order, viscous, bounds, deck, state builder, checkpoint steps)."""
    def vortex(X, g):
        return ics.isentropic_vortex(X, beta=5.0, gamma=g)

    def supersonic_vortex(X, g):
        # a weak vortex on a Mach 2 stream (p = rho = 1 far away: c = sqrt(gamma))
        return ics.isentropic_vortex(X, beta=0.5, u_inf=(2.0 * math.sqrt(g), 0.0), gamma=g)

    eul = {"mach_fs": 0.3, "rho_fs": 1.0, "P_fs": 1.0}
    return {
        # the vortex workload as specified: 32 x 32 quads on periodic [-5,5]^2,
        # P3, Rusanov, gamma 1.4, beta 5 vortex on a unit stream, RK44 with
        # dt 1e-3 for 1000 steps; the state is kept after 1, 10, 100 and 1000
        "quad_p3_vortex_32x32_rk44_1000": (lambda: meshgen.box_quads(32, 32), 2, 3, False,
                                           {"PERIODIC": "periodic"}, dict(eul, dt=1e-3), vortex, (1, 10, 100, 1000)),
        # supersonic inflow on the left, supersonic outflow on the right, slip
        # walls top and bottom; the vortex leaves through the outflow
        "quad_p2_supin_supout_slip": (lambda: meshgen.box_quads(8, 6, -1.0, 1.0, -0.75, 0.75,
                                                                bnd=("INFLOW", "OUTFLOW", "WALL", "WALL")),
                                      2, 2, False, {"INFLOW": "inlet_sup", "OUTFLOW": "outlet_sup", "WALL": "wall_slip"},
                                      {"mach_fs": 2.0, "rho_fs": 1.0, "P_fs": 1.0, "dt": 2e-3}, supersonic_vortex,
                                      (1, 10, 100, 200)),
    }


def make_traj_case(name, spec, tmp):
    """Reference RK44 trajectory: U0 and the state after each checkpoint step count."""
    build, ndims, order, viscous, bounds, deck, state_fn, checkpoints = spec
    mesh = build()
    meshgen.write_gmsh(mesh, os.path.join(tmp, name + ".msh"))
    deck_path = refcpu.write_deck(os.path.join(tmp, name + ".deck"), name + ".msh", ndims, order, viscous,
                                  bounds, deck)
    r = refcpu.RefSolver(deck_path)
    S, V, E = r.state_shape
    X = r.array("coord_spts").reshape(S, ndims, E)
    U0 = state_fn(X, r.params["gamma"])
    r.set_state(U0)
    states, done = [], 0
    for k in checkpoints:
        r.update(k - done)
        done = k
        states.append(r.get_state())
    faces_t = np.array([f[0] for f in mesh.bnd_faces], dtype=np.int64)
    npf = max((len(f[1]) for f in mesh.bnd_faces), default=1)
    faces_n = np.full((len(mesh.bnd_faces), npf), -1, dtype=np.int64)
    for i, f in enumerate(mesh.bnd_faces):
        faces_n[i, :len(f[1])] = f[1]
    faces_name = np.array([f[2] for f in mesh.bnd_faces])
    meta = {"name": name, "ndims": ndims, "order": order, "viscous": bool(viscous), "bounds": bounds,
            "deck": deck, "params": r.params, "checkpoints": list(checkpoints), "dt": r.params["dt"],
            "shape": [S, V, E], "gmsh_type": mesh.gmsh_type}
    os.makedirs(TRAJ_DIR, exist_ok=True)
    out = os.path.join(TRAJ_DIR, name + ".npz")
    np.savez_compressed(out, meta=json.dumps(meta), nodes=mesh.nodes, elements=mesh.elements, faces_type=faces_t,
                        faces_nodes=faces_n, faces_name=faces_name, U0=U0, states=np.array(states))
    r.close()
    return out


def main(names=None):
    with tempfile.TemporaryDirectory() as tmp:
        for table, fn in ((_cases(), make_case), (_time_cases(), make_time_case), (_cases(), make_diag_case),
                          (_traj_cases(), make_traj_case)):
            for name, spec in table.items():
                if names and name not in names:
                    continue
                out = fn(name, spec, tmp)
                print(f"{name}: {os.path.getsize(out) / 1024:.1f} KiB")


if __name__ == "__main__":
    main(sys.argv[1:])
