"""Reference input decks read by zefr_b200.deck: the parameters they give
(through zb_params_from_deck's non-dimensionalisation) equal the compiled
reference's own InputStruct values for the same deck file, and the
time-scheme and boundary keys come through.  CPU only."""
import os

import numpy as np
import pytest

from oracle import refcpu
from zefr_b200 import meshgen
from zefr_b200.deck import read_deck
from zefr_b200.solver import Plan, params_from_deck

FIELDS = ["gamma", "prandtl", "mu", "rt", "c_sth", "rus_k", "ldg_b", "ldg_tau", "rho_fs", "P_fs", "T_wall",
          "R_ref", "dt"]

CASES = {
    "euler_2d": (lambda: meshgen.box_quads(4, 4), 2, 3, False, {"PERIODIC": "periodic"},
                 {"mach_fs": 0.3, "rho_fs": 1.0, "P_fs": 1.0, "dt": 2e-3}),
    "tgv_3d_disable_nondim": (lambda: meshgen.box_hexes(2, 2, 2), 3, 3, True, {"PERIODIC": "periodic"},
                              {"disable_nondim": 1, "fix_vis": 1, "mach_fs": 0.1, "Re_fs": 1600, "prandtl": 0.71,
                               "P_fs": 1.0, "rho_fs": 1.0, "L_fs": 1.0, "ldg_b": 0.5, "ldg_tau": 0.1, "dt": 5e-4}),
    "cylinder_nondim_sutherland": (lambda: meshgen.cylinder_omesh(3, 8, r1=4.0), 2, 2, True,
                                   {"WALL": "wall_ns_iso", "FARFIELD": "char"},
                                   {"mach_fs": 0.2, "Re_fs": 100, "fix_vis": 0, "ldg_b": 0.3, "ldg_tau": 0.2,
                                    "T_wall": 320.0, "mach_wall": 0.05, "nx_wall": 0.6, "ny_wall": 0.8,
                                    "nx_fs": 0.8, "ny_fs": 0.6, "dt": 1e-4}),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_deck_parameters_match_reference(name, tmp_path):
    if not refcpu.available():
        pytest.skip("compiled reference not built (make -C oracle)")
    build, ndims, order, viscous, bounds, params = CASES[name]
    mesh = build()
    meshgen.write_gmsh(mesh, str(tmp_path / "m.msh"))
    deck = refcpu.write_deck(str(tmp_path / "case.deck"), "m.msh", ndims, order, viscous, bounds, params)
    r = refcpu.RefSolver(deck)
    ref = r.params
    r.close()
    d = read_deck(deck)
    assert d.meshfile == os.path.join(str(tmp_path), "m.msh")
    assert {k.lower(): v for k, v in d.bounds.items()} == {k.lower(): v for k, v in bounds.items()}
    p = params_from_deck(**d.params)
    assert p.order == order and p.viscous == int(viscous)
    assert p.fix_vis == int(ref["fix_vis"])
    for f in FIELDS:
        got, want = getattr(p, f), ref[f]
        assert abs(got - want) <= 1e-14 * max(abs(want), 1.0), (f, got, want)
    for i in range(3):
        assert abs(p.V_fs[i] - ref[f"V_fs{i}"]) <= 1e-14 * max(abs(ref[f"V_fs{i}"]), 1.0)
        assert abs(p.V_wall[i] - ref[f"V_wall{i}"]) <= 1e-14 * max(abs(ref[f"V_wall{i}"]), 1.0)
    plan = Plan(d.meshfile, p, d.bounds)
    assert plan.info.n_eles == len(mesh.elements)


def test_deck_time_scheme_and_flux_keys(tmp_path):
    path = tmp_path / "rk54.deck"
    path.write_text("\n".join([
        "nDims 2", "meshfile m.msh", "order 3", "viscous 0  # inviscid", "fconv_type Roe", "dt_scheme RK54",
        "dt 0.01", "adapt_dt 1", "err_atol 1e-6", "err_rtol 2e-6", "max_factor 2.0", "n_steps 7",
        "write_paraview 0", "mesh_bound fluid fluid", "mesh_bound PERIODIC periodic", ""]))
    d = read_deck(str(path))
    assert d.params["fconv"] == 2 and d.params["order"] == 3 and d.params["viscous"] == 0
    assert d.dt_scheme == "RK54" and d.n_steps == 7
    assert d.time_scheme == {"adapt_dt": 1, "err_atol": 1e-6, "err_rtol": 2e-6, "max_factor": 2.0}
    assert d.bounds == {"PERIODIC": "periodic"}
    assert d.raw["write_paraview"] == "0"


@pytest.mark.parametrize("line", ["equation AdvDiff", "fvisc_type Central", "spt_type Lobatto",
                                  "dt_scheme DIRK34", "fconv_type HLLC"])
def test_deck_rejects_unbuilt_options(tmp_path, line):
    path = tmp_path / "bad.deck"
    path.write_text("nDims 2\nmeshfile m.msh\norder 2\n" + line + "\n")
    with pytest.raises(ValueError):
        read_deck(str(path))


def test_deck_requires_core_keys(tmp_path):
    path = tmp_path / "short.deck"
    path.write_text("nDims 2\norder 2\n")
    with pytest.raises(ValueError):
        read_deck(str(path))
