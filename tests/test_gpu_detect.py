"""Proximity detection on the GPU (cs_detect_proximities) against the CPU oracle's
restatement of Simulator::findProximities, which is itself pinned bit for bit to the
reference's own predicates (tests/test_oracle.py).

Bars: the same proximities in the same order (node ids exact; normals, weights, stiffness and
friction bit for bit, both sides computing the reference's FP32 expressions in its order);
detection + step against the oracle doing the same per cloth, dv to 1e-6 of the FP64 solve;
deterministic repeat; collision groups; a non-finite state reported as an argument error.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import proxutil
import pyoracle
from clothsimulator_b200 import native, scenes

REP = 1e-3  # Magic::repulsionThickness default


def oracle_cloths(scene):
    return [pyoracle.Cloth(s, pyoracle.Material(s["material"], "float")) for s in scene.sheets]


def params_for(scene, **kw):
    kw.setdefault("tol", 1e-10)
    kw.setdefault("max_iters", 20000)
    return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, **kw)


def assert_same(gpu, ora):
    n = len(ora["mu"])
    assert len(gpu["mu"]) == n and n > 0
    assert np.array_equal(gpu["nodes"], ora["nodes"])
    for k in ("normal", "w", "mu", "stiffness"):
        assert np.array_equal(gpu[k], ora[k].astype(np.float32)), k


@pytest.mark.parametrize("make", [lambda: scenes.folded_sheet(16), lambda: scenes.stacked_sheets(12, n_layers=3)],
                         ids=["folded16", "stacked3x12"])
def test_detection_matches_oracle(ctx_factory, make):
    scene = make()
    ctx = ctx_factory(scene.sheets)
    n = ctx.detect_proximities(REP)
    ora = pyoracle.detect_proximities(oracle_cloths(scene), repulsion_thickness=REP)
    assert n == len(ora["mu"])
    assert_same(ctx.get_proximities(), ora)
    assert set(np.unique(ora["kind"])) == {0, 1, 2}


def test_detection_is_deterministic(ctx_factory):
    scene = scenes.stacked_sheets(16, n_layers=2, seed=3)
    ctx = ctx_factory(scene.sheets)
    ctx.detect_proximities(REP)
    a = ctx.get_proximities()
    ctx.detect_proximities(REP)
    b = ctx.get_proximities()
    for k in a:
        assert np.array_equal(a[k], b[k])


def test_collision_groups(ctx_factory):
    """Stacked layers in separate groups see no proximities (flat layers have none of their
    own); a batch of two independent stacks finds each stack's own."""
    one = scenes.stacked_sheets(12, n_layers=2, seed=5)
    ctx = ctx_factory(one.sheets)
    assert ctx.detect_proximities(REP, groups=[0, 1]) == 0
    two = scenes.Scene("two_stacks", one.sheets + scenes.stacked_sheets(12, n_layers=2, seed=6).sheets, one.dt, 1)
    ctx2 = ctx_factory(two.sheets)
    ctx2.detect_proximities(REP, groups=[0, 0, 1, 1])
    got = ctx2.get_proximities()
    cl = oracle_cloths(two)
    ora = pyoracle.detect_proximities(cl, groups=[0, 0, 1, 1], repulsion_thickness=REP)
    assert_same(got, ora)
    offs = proxutil.offsets(two)
    # no proximity couples the stacks
    stack = (got["nodes"] >= offs[2]).astype(int)
    assert np.all(stack.min(axis=1) == stack.max(axis=1))


def test_detect_then_step_matches_oracle(ctx_factory):
    scene = scenes.folded_sheet(16, seed=2)
    ctx = ctx_factory(scene.sheets)
    ctx.detect_proximities(REP)
    stats, _ = ctx.step(params_for(scene, advance=0))
    assert stats.converged == 1 and stats.max_rel_residual <= 1e-10
    cl = oracle_cloths(scene)
    ora = pyoracle.detect_proximities(cl, repulsion_thickness=REP)
    proxutil.set_oracle_proximities(cl, ora, proxutil.offsets(scene), REP)
    cl[0].assemble(scenes.step_params(scene, scene.sheets[0]))
    odv, _ = cl[0].solve(pyoracle.METHOD_LLT64)
    dv = ctx.get_dv().reshape(-1)
    assert np.linalg.norm(dv - odv) / np.linalg.norm(odv) < 1e-6


def test_simulation_with_detection_tracks_oracle(ctx_factory):
    """Three reference-style steps (detect, then step) of two stacked sheets, GPU against the
    oracle cloths: the same proximities every step, positions within 1e-5 of the step."""
    scene = scenes.stacked_sheets(12, n_layers=2, seed=7)
    offs = proxutil.offsets(scene)
    ctx = ctx_factory(scene.sheets)
    cl = oracle_cloths(scene)
    x0 = np.concatenate([s["x"] for s in scene.sheets]).astype(np.float64)
    for _ in range(3):
        ctx.detect_proximities(REP)
        ora = pyoracle.detect_proximities(cl, repulsion_thickness=REP)
        got = ctx.get_proximities()
        assert np.array_equal(got["nodes"], ora["nodes"])
        proxutil.set_oracle_proximities(cl, ora, offs, REP)
        for k, c in enumerate(cl):
            c.step(scenes.step_params(scene, scene.sheets[k]), pyoracle.METHOD_LLT64)
        stats, _ = ctx.step(params_for(scene))
        assert stats.converged == len(scene.sheets)
        # carry the oracle's state forward from the GPU's, so each step compares one step
        x, v = ctx.get_state()
        xo = np.concatenate([c.state()[0] for c in cl])
        d = xo - x0.reshape(-1, 3)
        assert np.linalg.norm(x.reshape(-1, 3) - xo) / np.linalg.norm(d) < 1e-5
        o = 0
        for c in cl:
            m = c.n
            c.set_state(x.reshape(-1, 3)[o:o + m], v.reshape(-1, 3)[o:o + m])
            o += m
        x0 = x.astype(np.float64)


def test_non_finite_state_is_reported(ctx_factory):
    scene = scenes.folded_sheet(8, seed=4)
    ctx = ctx_factory(scene.sheets)
    x = scene.sheets[0]["x"].copy()
    x[3, 1] = np.nan
    ctx.set_state(x)
    with pytest.raises(native.ClothStepError) as e:
        ctx.detect_proximities(REP)
    assert e.value.status == native.CS_ERR_INVALID_ARG
