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


def test_coplanar_start_matches_oracle(ctx_factory):
    """Impacts at t = 0 exactly: one row of the upper layer starts in the plane of the lower
    layer (both at z = 0), the rest 1.5 mm above, and the layer moves up 1 mm.  The quadratic's
    c / q gives some of those times as -0.0, which the order of impacts (time, then node ids,
    type, index) must take as equal to +0.0, as the oracle's comparison does.  A start that is
    coplanar stays coplanar in every round (x0 does not move), so both sides give up after
    2 x 100 rounds, with the same impacts chosen and projected in each round."""
    scene = scenes.stacked_sheets(6, n_layers=2, seed=7)
    n = 7
    for k, s in enumerate(scene.sheets):
        s["x"] = s["x"].copy()
        s["x"][:, 2] = 0.0 if k == 0 else 1.5e-3
        if k == 1:
            s["x"][2 * n:3 * n, 2] = 0.0
    xs = dropped(scene, lambda k, x: np.full(len(x), k == 1), -1e-3)
    ctx = ctx_factory(scene.sheets)
    ctx.set_state(np.concatenate(xs), np.zeros((sum(len(x) for x in xs), 3), np.float32))
    rounds, impacts, st = ctx.collision_step(DT, allow_unresolved=True)
    x, _ = ctx.get_state()
    cl = oracle_cloths(scene)
    for c, xe in zip(cl, xs):
        c.set_state(xe.astype(np.float64), np.zeros(xe.shape))
    orounds, oimpacts = pyoracle.collision_step(cl, DT)
    ox = np.concatenate([c.state()[0] for c in cl])
    assert orounds == -1 and st == native.CS_ERR_NOT_CONVERGED
    assert oimpacts > 0 and impacts == oimpacts
    assert np.array_equal(x.reshape(-1, 3), ox.astype(np.float32))


def test_impact_order_ties_and_signed_zero(ctx_factory):
    """The collision step's device sort of a round's impacts (cs_impact_order: four stable radix
    passes over type, (n2, n3), n1, (t, n0)) equals the oracle's order -- time with -0.0 equal
    to +0.0 (impactBefore, oracle_collide.hpp), then node ids, then type -- with the input index
    as the last key, on records built to tie: few distinct times, small node ids, both types,
    exact duplicates."""
    scene = scenes.hang(8)
    ctx = ctx_factory(scene.sheets)
    rng = np.random.default_rng(3)
    n = 3000
    t = rng.choice(np.array([0.0, -0.0, 0.25, 0.5, 0.5000001, 1.0], np.float32), n)
    nodes = rng.integers(0, 5, size=(n, 4)).astype(np.int32)
    types = rng.integers(0, 2, n).astype(np.int32)
    nodes[100:110] = nodes[99]
    t[100:110] = t[99]
    types[100:110] = types[99]
    order = ctx.impact_order(nodes, t, types)
    ref = sorted(range(n), key=lambda i: (float(t[i]) + 0.0, *(int(v) for v in nodes[i]), int(types[i]), i))
    assert np.array_equal(order, np.array(ref, np.int32))
    assert np.any(np.signbit(t) & (t == 0)) and np.any(~np.signbit(t) & (t == 0))
