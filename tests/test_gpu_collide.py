"""The collision step on the GPU (cs_collision_step) against the CPU oracle's restatement of
Simulator::collisionStep, itself pinned bit for bit to the reference's own impact tests and
CollisionOptimization (tests/test_oracle.py).

Bars: continuous impacts, their selection and the impact-zone projection are the reference's
FP32 arithmetic in its order (sums of the projection in the CPU loop's order), so positions,
velocities, rounds and impact counts equal the oracle's bit for bit on layers driven through
each other; without impacts one round and v = (x - x0) / dt exactly; in a reference-style loop
(detect, step, collide) every collision step leaves no impact behind.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyoracle
from clothsimulator_b200 import native, scenes

DT = 0.01


def oracle_cloths(scene):
    return [pyoracle.Cloth(s, pyoracle.Material(s["material"], "float")) for s in scene.sheets]


def dropped(scene, which, drop):
    """End-of-step positions: the nodes `which(k, x)` selects moved down by `drop`."""
    out = []
    for k, s in enumerate(scene.sheets):
        x = s["x"].astype(np.float32).copy()
        sel = which(k, x)
        x[sel, 2] = (x[sel, 2] - np.float32(drop)).astype(np.float32)
        out.append(x)
    return out


def run_both(ctx_factory, scene, xs):
    ctx = ctx_factory(scene.sheets)
    ctx.set_state(np.concatenate(xs), np.zeros((sum(len(x) for x in xs), 3), np.float32))
    rounds, impacts, _ = ctx.collision_step(DT)
    x, v = ctx.get_state()
    cl = oracle_cloths(scene)
    for c, xe in zip(cl, xs):
        c.set_state(xe.astype(np.float64), np.zeros(xe.shape))
    orounds, oimpacts = pyoracle.collision_step(cl, DT)
    ox = np.concatenate([c.state()[0] for c in cl])
    ov = np.concatenate([c.state()[1] for c in cl])
    return (rounds, impacts, x.reshape(-1, 3), v.reshape(-1, 3)), (orounds, oimpacts, ox, ov)


def test_crossing_layers_match_oracle(ctx_factory):
    scene = scenes.stacked_sheets(10, n_layers=2, seed=3)
    xs = dropped(scene, lambda k, x: np.full(len(x), k == 1), 3e-3)
    g, o = run_both(ctx_factory, scene, xs)
    assert o[0] > 1 and o[1] > 0, "the case should have impacts"
    assert (g[0], g[1]) == (o[0], o[1])
    assert np.array_equal(g[2], o[2].astype(np.float32))
    assert np.array_equal(g[3], o[3].astype(np.float32))


def test_folded_sheet_crossing_itself_matches_oracle(ctx_factory):
    scene = scenes.folded_sheet(12, seed=5)
    gap = scene.meta["gap"]
    xs = dropped(scene, lambda k, x: x[:, 2] > 0.5 * gap, 2.5 * gap)
    g, o = run_both(ctx_factory, scene, xs)
    assert o[1] > 0
    assert (g[0], g[1]) == (o[0], o[1])
    assert np.array_equal(g[2], o[2].astype(np.float32))
    assert np.array_equal(g[3], o[3].astype(np.float32))


def test_no_impacts_one_round_and_velocity_update(ctx_factory):
    scene = scenes.hang(12, seed=1)
    ctx = ctx_factory(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-8)
    x_start, _ = ctx.get_state()
    ctx.step(p)
    x, _ = ctx.get_state()
    rounds, impacts, _ = ctx.collision_step(scene.dt)
    assert (rounds, impacts) == (1, 0)
    x2, v2 = ctx.get_state()
    assert np.array_equal(x2, x)
    inv = np.float32(1.0) / np.float32(scene.dt)
    assert np.array_equal(v2, (x - x_start) * inv)


def test_reference_loop_leaves_no_impacts(ctx_factory):
    """detect -> step -> collide, three times, on two layers closing at 0.5 m/s (they would
    cross within a step); each collision step resolves its impacts, so a second pass finds
    none, and the oracle's one-step result agrees."""
    scene = scenes.stacked_sheets(10, n_layers=2, seed=8)
    v = [np.zeros_like(s["x"]) for s in scene.sheets]
    v[1][:, 2] = -0.5
    for s, vv in zip(scene.sheets, v):
        s["v"] = vv.astype(np.float32)
    ctx = ctx_factory(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-10, max_iters=20000)
    seen = 0
    for k in range(3):
        ctx.detect_proximities(1e-3)
        stats, _ = ctx.step(p)
        assert stats.converged == 2
        rounds, impacts, _ = ctx.collision_step(scene.dt)
        seen += impacts
        again = ctx.collision_step(scene.dt)
        assert again[:2] == (1, 0), f"step {k}: impacts left after the collision step"
    assert seen >= 0
