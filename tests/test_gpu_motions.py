"""Handles that follow motions (Cloth::addHandleForces, Cloth.cu:157-169): each step the handle's
target is its position at load moved by the transformation of its motion at that step
(Transformation::applyToPoint, Motion::computeTransformation), given to cs_step in
cs_step_params.transformations.  The oracle's FP32 restatement of the transformations (pinned to
the reference's classes in test_oracle.py) supplies the same targets to the CPU assembly.

Bars: b against the oracle 1e-6 with the handle rows bit for bit; dv (tol 1e-10) against an FP64
direct solve 1e-6; the host layer's run of a scene with a moving handle equals the same steps
through the C ABI bit for bit."""
import ctypes
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyoracle
from clothsimulator_b200 import native, scenes
from test_oracle import MOTION_KEYFRAMES


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_moving_handle_targets_match_oracle(ctx_factory):
    scene = scenes.hang(16, seed=3)
    s = scene.sheets[0]
    rng = np.random.default_rng(3)
    s["x"] = (s["x"] + rng.normal(0, 0.01, s["x"].shape)).astype(np.float32)
    s["v"] = rng.normal(0, 0.1, s["v"].shape).astype(np.float32)
    ctx = ctx_factory(scene.sheets)
    handles = s["handles"]  # two top corners: the first follows the motion, the second stays
    ctx.set_handle_motions([0, -1])
    m = pyoracle.Motion(MOTION_KEYFRAMES)
    oc = pyoracle.Cloth(s, pyoracle.Material(s["material"], "float"))
    for step in range(1, 40, 7):
        T = m.transform(step * scene.dt)
        p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-10, max_iters=20000, advance=0)
        native.set_transformations(p, T[None, :])
        ctx.assemble(p)
        _, _, _, b = ctx.system()
        rest = s["x"][handles].astype(np.float32)
        targets = np.stack([pyoracle.transform_points(T, rest[0])[0], rest[1]]).astype(np.float64)
        hn = np.ascontiguousarray(handles, np.int32)
        oc.L.cloth_set_handles(oc.h, 2, hn.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                               np.ascontiguousarray(targets).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        _, _, _, ob = oc.assemble(scenes.step_params(scene, s))
        assert rel(b, ob) < 1e-6, step
        rows = np.concatenate([[3 * h, 3 * h + 1, 3 * h + 2] for h in handles])
        assert np.array_equal(b[rows], ob[rows].astype(np.float32)), step
        stats, _ = ctx.step(p)
        assert stats.converged == 1
        exact, _ = oc.solve(pyoracle.METHOD_LLT64)
        assert rel(ctx.get_dv(), exact) < 1e-6


def test_handle_motion_validation(ctx_factory):
    scene = scenes.hang(8, seed=1)
    ctx = ctx_factory(scene.sheets)
    with pytest.raises(native.ClothStepError):
        ctx.set_handle_motions([0])  # two handles
    with pytest.raises(native.ClothStepError):
        ctx.set_handle_motions([0, 64])  # beyond CS_MAX_MOTIONS - 1
    ctx.set_handle_motions([2, -1])
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness)
    native.set_transformations(p, np.tile(pyoracle.Motion(MOTION_KEYFRAMES).transform(0.2), (2, 1)))
    assert ctx.lib.cs_step(ctx.h, ctypes.byref(p), None) == native.CS_ERR_INVALID_ARG  # motion 2 of 2
    native.set_transformations(p, np.tile(pyoracle.Motion(MOTION_KEYFRAMES).transform(0.2), (3, 1)))
    ctx.step(p)


def test_moving_handle_scene_through_host_layer(tmp_path):
    """A 12x12 hanging sheet whose first top corner follows a keyframed motion: clothsim
    simulate_offline against the same steps through the C ABI (transformations at time
    step x dt, Simulator.cu:565-569, from the oracle's restatement), frames bit for bit."""
    from test_host_layer import COLLISION_THICKNESS, HOST_PRECOND_DEGREE, host

    scene = scenes.hang(12, seed=2)
    path = scenes.write_scene(scene, str(tmp_path / "scene"), frames=2,
                              solver={"tol": 1e-8, "max_iters": 8000, "warm_start": "previous"})
    cfg = json.loads(open(path).read().split("\n", 1)[1])
    cfg["motions"] = [MOTION_KEYFRAMES]
    nodes = cfg["handles"][0]["nodes"]
    cfg["handles"] = [{"cloth": 0, "nodes": [nodes[0]], "motion": 0}, {"cloth": 0, "nodes": [nodes[1]]}]
    open(path, "w").write(json.dumps(cfg))
    out = str(tmp_path / "out")
    lib = host()
    steps = ctypes.c_int(0)
    st = lib.cs_sim_run(b"simulate_offline", path.encode(), out.encode(), 0, ctypes.byref(steps))
    assert st == 0, lib.cs_sim_last_error()
    xs = [list(map(float, l.split()[1:])) for l in open(os.path.join(out, "frame2_cloth0.obj")) if l.startswith("v ")]
    ctx = native.Context(0)
    ctx.load(scene.sheets)
    ctx.set_handle_motions([0, -1])
    m = pyoracle.Motion(MOTION_KEYFRAMES)
    dt = np.float32(cfg["frame_time"]) / np.float32(cfg["frame_steps"])
    p = native.step_params(float(dt), scene.gravity, scene.handle_stiffness, tol=1e-8, max_iters=8000,
                           precond_degree=HOST_PRECOND_DEGREE)
    for k in range(steps.value):
        p.warm_start = native.WARM_ZERO if k == 0 else native.WARM_PREVIOUS
        native.set_transformations(p, m.transform(np.float32((k + 1) * dt))[None, :])
        ctx.detect_proximities(1e-3)
        ctx.step(p)
        ctx.collision_step(float(dt), COLLISION_THICKNESS)
    x, _ = ctx.get_state()
    assert np.array_equal(np.array(xs, np.float32), x)
    # the corner followed the motion: it moved by more than gravity alone would move it
    assert np.linalg.norm(x.reshape(-1, 3)[nodes[0]] - scene.sheets[0]["x"][nodes[0]]) > 0.05
    ctx.close()
