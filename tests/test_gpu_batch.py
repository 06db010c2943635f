"""Batched persistent stages: every case of a batch must advance as it does
stepped alone (the batch runs the single-case tile body: identical in FP64,
and within FP32 rounding in the mixed form, where the compiler may contract
multiply-adds differently in the two kernels), with or without the CUDA
graph, and the autotuner must leave the states untouched."""
import numpy as np
import pytest

from zefr_b200 import batch as zbatch

pytestmark = pytest.mark.gpu


def _same(a, b, precision):
    if precision == "fp64":
        return np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
    return np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


def _pair(precision, seed=5, n=10):
    a = zbatch.vortex_cases(n, seed, n_range=(3, 9), precision=precision)
    b = zbatch.vortex_cases(n, seed, n_range=(3, 9), precision=precision)
    return a, b


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_cases_stepped_alone(precision, graph):
    alone, batched = _pair(precision)
    assert len({s.case["P"] for s in alone}) >= 3
    for s in alone:
        s.step(3)
    bt = zbatch.Batch(batched)
    bt.step(3, graph=graph)
    bt.synchronize()
    for s1, s2 in zip(alone, batched):
        assert _same(s1.get_state(), s2.get_state(), precision)


@pytest.mark.parametrize("shape", [(256, 256, 1), (128, 64, 1), (64, 64, 1), (256, 64, 8), (128, 128, 32), (256, 64, 0)])
def test_batch_launch_shapes_agree(shape):
    """Whole-CTA tiles (one group) and several tile groups per CTA (named
    barriers) compute the same stages."""
    alone, batched = _pair("fp64", seed=13, n=7)
    for s in alone:
        s.step(2)
    bt = zbatch.Batch(batched)
    bt.set_config(threads=shape[0], blocks_per_sm=3, order=0, group=shape[1], chunk=shape[2])
    bt.step(2)
    bt.synchronize()
    for s1, s2 in zip(alone, batched):
        assert _same(s1.get_state(), s2.get_state(), "fp64")


def test_batch_single_stages_match():
    alone, batched = _pair("fp64", seed=9, n=6)
    bt = zbatch.Batch(batched)
    for st in range(4):
        bt.stage(st)
        for s in alone:
            s.step_RK_stage(st)
    for s1, s2 in zip(alone, batched):
        assert _same(s1.get_state(), s2.get_state(), "fp64")


def test_autotune_keeps_state_and_picks_a_shape():
    cases = zbatch.vortex_cases(8, 3, n_range=(4, 12), precision="mixed")
    before = [s.get_state() for s in cases]
    bt = zbatch.Batch(cases)
    cfg = bt.autotune(steps=2)
    assert cfg["threads"] in (64, 128, 256) and cfg["threads"] % cfg["group"] == 0
    assert cfg["blocks_per_sm"] >= 1 and cfg["ms_per_step"] > 0
    for s, u in zip(cases, before):
        assert np.array_equal(s.get_state(), u)
    # stepping after tuning still matches the cases stepped alone
    ref = zbatch.vortex_cases(8, 3, n_range=(4, 12), precision="mixed")
    for s in ref:
        s.step(2)
    bt.step(2)
    bt.synchronize()
    for s1, s2 in zip(ref, cases):
        assert _same(s1.get_state(), s2.get_state(), "mixed")


@pytest.mark.parametrize("form", [True, False])
def test_autotune_of_one_form_installs_that_form(form):
    """Tuning restricted to one form picks a shape of that form, leaves the
    states untouched, and the installed shape steps as the cases do alone."""
    cases = zbatch.vortex_cases(8, 7, n_range=(4, 12), precision="mixed")
    before = [s.get_state() for s in cases]
    bt = zbatch.Batch(cases)
    cfg = bt.autotune(steps=1, form=form)
    assert cfg["fused"] == int(form) and cfg["ms_per_step"] > 0
    for s, u in zip(cases, before):
        assert np.array_equal(s.get_state(), u)
    orders = len({c.info.order for c in cases})
    n0 = bt.launch_count()
    bt.step(2)
    bt.synchronize()
    assert bt.launch_count() - n0 == 2 * 4 * (1 if form else orders)
    ref = zbatch.vortex_cases(8, 7, n_range=(4, 12), precision="mixed")
    for s in ref:
        s.step(2)
    for s1, s2 in zip(ref, cases):
        assert _same(s1.get_state(), s2.get_state(), "mixed")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(256, 64, 0), (128, 128, 1), (256, 256, 8)])
def test_fused_single_launch_matches_cases_stepped_alone(precision, shape):
    """One persistent launch per stage for every order present: the same
    stages as the cases stepped alone, four launches per step."""
    alone, batched = _pair(precision, seed=21, n=9)
    orders = len({s.case["P"] for s in alone})
    assert orders >= 3
    for s in alone:
        s.step(3)
    bt = zbatch.Batch(batched)
    bt.set_config(threads=shape[0], blocks_per_sm=2, order=0, group=shape[1], chunk=shape[2], fused=True)
    n0 = bt.launch_count()
    bt.step(3)
    bt.synchronize()
    assert bt.launch_count() - n0 == 3 * 4
    for s1, s2 in zip(alone, batched):
        assert _same(s1.get_state(), s2.get_state(), precision)


def test_graph_is_one_replay_of_one_launch_per_order_and_stage():
    cases = zbatch.vortex_cases(4, 1, n_range=(3, 5), precision="mixed")
    orders = len({c.info.order for c in cases})
    bt = zbatch.Batch(cases)
    n0 = bt.launch_count()
    bt.step(5)
    bt.synchronize()
    assert bt.launch_count() - n0 == 5 * 4 * orders


def test_batch_rejects_viscous_and_hex():
    from zefr_b200 import meshgen
    from zefr_b200.solver import FRSolver, make_params
    from zefr_b200._lib import ZbError
    s = FRSolver(meshgen.box_quads(3, 3), make_params(2, True, mu=1e-3), {"PERIODIC": "periodic"})
    with pytest.raises(ZbError):
        zbatch.Batch([s])
    h = FRSolver(meshgen.box_hexes(2, 2, 2), make_params(2, False), {"PERIODIC": "periodic"})
    with pytest.raises(ZbError):
        zbatch.Batch([h])
