"""C ABI of libzefr_b200.so on the CPU: the library loads, exports every entry
point include/zb.h declares, and host-side set-up errors come back as status
codes with a message (no GPU calls here)."""
import ctypes
import os
import re

import numpy as np
import pytest

from zefr_b200 import _lib, meshgen
from zefr_b200.solver import Plan, make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "zb.h")).read()
    return sorted(set(re.findall(r"\b(zb_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(syms) == sorted(_lib.EXPORTED)


def test_version_string():
    assert b"sm_100a" in _lib.lib().zb_version()


def _err(fn):
    with pytest.raises(_lib.ZbError) as ei:
        fn()
    return ei.value


def test_unpaired_periodic_face():
    m = meshgen.box_quads(3, 3)
    # move one boundary node so a periodic face loses its partner
    nodes = m.nodes.copy()
    nodes[1, 0] += 0.3
    m.nodes = nodes
    e = _err(lambda: Plan(m, make_params(2), {"PERIODIC": "periodic"}))
    assert e.status == -3 and "periodic" in str(e).lower()


def test_negative_jacobian():
    m = meshgen.box_quads(2, 2)
    m.elements = m.elements[:, ::-1].copy()
    e = _err(lambda: Plan(m, make_params(2), {"PERIODIC": "periodic"}))
    assert e.status == -3 and "Jacobian" in str(e)


def test_unknown_boundary_name():
    m = meshgen.box_quads(2, 2)
    with pytest.raises(ValueError):
        Plan(m, make_params(2), {"WALL": "wall_slip"})


def test_gmsh_reader_errors(tmp_path):
    m = meshgen.box_quads(2, 2)
    p = str(tmp_path / "m.msh")
    meshgen.write_gmsh(m, p)
    out = ctypes.POINTER(_lib.ZbMesh)()
    names = (ctypes.c_char_p * 1)(b"nothing")
    bcs = (ctypes.c_int * 1)(1)
    st = _lib.lib().zb_mesh_read_gmsh(p.encode(), 2, 1, names, bcs, ctypes.byref(out))
    assert st == -3 and b"Unrecognized mesh boundary" in _lib.lib().zb_last_error()
    names = (ctypes.c_char_p * 1)(b"periodic")
    st = _lib.lib().zb_mesh_read_gmsh(p.encode(), 2, 1, names, bcs, ctypes.byref(out))
    assert st == 0
    assert out.contents.n_eles == 4 and out.contents.gmsh_type == 3 and out.contents.n_bnd_faces == 8
    _lib.lib().zb_mesh_free(out)
    st = _lib.lib().zb_mesh_read_gmsh(str(tmp_path / "missing.msh").encode(), 2, 1, names, bcs, ctypes.byref(out))
    assert st == -1


def test_unsupported_element_and_order():
    m = meshgen.box_tris(2, seed=0, jitter=0.0)
    Plan(m, make_params(8), {"PERIODIC": "periodic"})  # triangles P1-P8 are built
    e = _err(lambda: Plan(m, make_params(9), {"PERIODIC": "periodic"}))
    assert e.status == -4
    e = _err(lambda: Plan(meshgen.box_quads(2, 2), make_params(12), {"PERIODIC": "periodic"}))
    assert e.status == -4


def test_plan_get_unknown_and_null():
    plan = Plan(meshgen.box_quads(2, 2), make_params(1), {"PERIODIC": "periodic"})
    with pytest.raises(_lib.ZbError):
        plan.get("no_such_array")
    assert _lib.lib().zb_plan_create(None, None, None) == -1
    assert _lib.lib().zb_compute_residual(None, 0) == -1


def test_params_from_deck_matches_reference_nondim():
    from zefr_b200.solver import params_from_deck
    p = params_from_deck(ndims=3, order=3, viscous=1, disable_nondim=1, fix_vis=1, mach_fs=0.1, Re_fs=1600,
                         P_fs=1.0, rho_fs=1.0, L_fs=1.0, gamma=1.4)
    c = np.sqrt(1.4)
    assert abs(p.V_fs[0] - 0.1 * c) < 1e-15
    assert abs(p.mu - 0.1 * c / 1600) < 1e-17


def test_adjoint_and_geometry_entry_points_reject_a_null_context():
    """The step adjoint and geometry entry points check their context before
    touching the GPU: a null one is ZB_ERR_ARG with a message, no crash."""
    L = _lib.lib()
    calls = {
        "zb_rk_step_vjp": lambda: L.zb_rk_step_vjp(None, None, None, None, 1, 1, 1, _lib.ZB_HOST, None, 0),
        "zb_geometry_eval": lambda: L.zb_geometry_eval(None, None, None, None, None, None, _lib.ZB_HOST),
        "zb_geometry_eval_vjp": lambda: L.zb_geometry_eval_vjp(None, None, None, None, None, None, None,
                                                               _lib.ZB_HOST),
        "zb_set_nodes": lambda: L.zb_set_nodes(None, None, _lib.ZB_HOST),
    }
    for name, call in calls.items():
        assert call() == -1, name
        assert b"null" in L.zb_last_error(), name


def test_batch_tuning_entry_points_reject_a_null_batch():
    """Both autotuners check the batch before touching the GPU."""
    L = _lib.lib()
    cfg = _lib.ZbBatchConfig()
    assert L.zb_batch_autotune(None, 1, ctypes.byref(cfg)) == -1
    assert b"null" in L.zb_last_error()
    for form in (-1, 0, 1):
        assert L.zb_batch_autotune_form(None, 1, form, ctypes.byref(cfg)) == -1
        assert b"null" in L.zb_last_error()
