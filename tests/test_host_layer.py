"""The host scene layer (Simulator/Cloth/Material/Handle over the C ABI): scene parsing and
validation on the CPU, and a headless run on the GPU compared with the C ABI driven directly."""
import ctypes
import json
import os

import numpy as np
import pytest

from clothsimulator_b200 import native, scenes

LIB = os.path.join(os.path.dirname(native.LIB_PATH), "libclothsim.so")


def host():
    lib = ctypes.CDLL(LIB)
    lib.cs_scene_describe.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.cs_sim_run.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                               ctypes.POINTER(ctypes.c_int)]
    lib.cs_sim_last_error.restype = ctypes.c_char_p
    return lib


def describe(path):
    lib = host()
    counts = (ctypes.c_longlong * 4)()
    st = lib.cs_scene_describe(path.encode(), counts)
    return st, list(counts), lib.cs_sim_last_error().decode()


def test_scene_description_matches_generator(tmp_path):
    scene = scenes.uneven_batch(3, seed=4, nq_range=(5, 9))
    path = scenes.write_scene(scene, str(tmp_path))
    st, counts, err = describe(path)
    assert st == 0, err
    assert counts == [3, scene.n_nodes, scene.n_faces, sum(len(s["handles"]) for s in scene.sheets)]


def test_quad_faces_are_triangulated(tmp_path):
    obj = tmp_path / "quad.obj"
    obj.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    mat = scenes.write_material_file(scenes.isotropic_material(10, 1e-5), str(tmp_path), "m")
    cfg = tmp_path / "c.json"
    cfg.write_text(json.dumps({"frame_time": 0.04, "frame_steps": 4, "cloths": [{"mesh": str(obj),
                   "materials": {"data": mat}}], "disable": ["remeshing"]}))
    st, counts, err = describe(str(cfg))
    assert st == 0, err
    assert counts == [1, 4, 2, 0]


@pytest.mark.parametrize("mutate,needle", [
    (lambda c: c.pop("disable"), "remeshing"),
    (lambda c: c.__setitem__("obstacles", [{"mesh": "ball.obj"}]), "obstacles"),
    (lambda c: c["handles"][0]["nodes"].append(10 ** 6), "out of range"),
    (lambda c: c["handles"][0].__setitem__("motion", 0), "motions"),
])
def test_unsupported_or_invalid_scenes_are_rejected(tmp_path, mutate, needle):
    scene = scenes.hang(4, seed=0)
    path = scenes.write_scene(scene, str(tmp_path))
    cfg = json.loads(open(path).read().split("\n", 1)[1])
    mutate(cfg)
    open(path, "w").write(json.dumps(cfg))
    st, _, err = describe(path)
    assert st == native.CS_ERR_INVALID_ARG and needle in err


def test_malformed_json_is_rejected(tmp_path):
    p = tmp_path / "bad.json"
    p.write_text('{"frame_time": 0.04, "cloths": [ }')
    st, _, err = describe(str(p))
    assert st == native.CS_ERR_INVALID_ARG and "JSON" in err


def test_interactive_modes_report_unavailable():
    lib = host()
    for mode in (b"simulate", b"resume", b"replay"):
        assert lib.cs_sim_run(mode, b"x", b"y", 0, None) == native.CS_ERR_INVALID_ARG
        assert b"unavailable" in lib.cs_sim_last_error()


# Magic::collisionThickness default, computed as the host layer does: 0.1f x repulsionThickness
# (Magic.cu:9-16) in FP32
COLLISION_THICKNESS = float(np.float32(0.1) * np.float32(1e-3))
# the host layer's default solver.precond_degree (SolverOptions::precondDegree)
HOST_PRECOND_DEGREE = 3


@pytest.mark.gpu
def test_simulate_offline_matches_c_abi(tmp_path):
    scene = scenes.hang(12, seed=2)
    path = scenes.write_scene(scene, str(tmp_path / "scene"), frames=2,
                              solver={"tol": 1e-8, "max_iters": 8000, "warm_start": "previous"})
    out = str(tmp_path / "out")
    lib = host()
    steps = ctypes.c_int(0)
    st = lib.cs_sim_run(b"simulate_offline", path.encode(), out.encode(), 0, ctypes.byref(steps))
    assert st == 0, lib.cs_sim_last_error()
    assert steps.value == 8 and os.path.exists(os.path.join(out, "frame2_cloth0.obj"))
    xs = [list(map(float, l.split()[1:])) for l in open(os.path.join(out, "frame2_cloth0.obj")) if l.startswith("v ")]
    # the same scene through the C ABI directly (OBJ text has 20 significant digits: exact floats)
    ctx = native.Context(0)
    ctx.load(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-8, max_iters=8000,
                           precond_degree=HOST_PRECOND_DEGREE)
    for k in range(8):
        p.warm_start = native.WARM_ZERO if k == 0 else native.WARM_PREVIOUS
        ctx.detect_proximities(1e-3)  # the host layer detects before every step, as Simulator.cu:571-586
        ctx.step(p)
        ctx.collision_step(scene.dt, COLLISION_THICKNESS)  # and the collision step after it (Simulator.cu:602-684)
    x, _ = ctx.get_state()
    assert np.array_equal(np.array(xs, np.float32), x)
    # resume continues from the last frame
    cfg = json.load(open(os.path.join(out, "config.json")))
    cfg["end_frame"] = 3
    json.dump(cfg, open(os.path.join(out, "config.json"), "w"))
    st = lib.cs_sim_run(b"resume_offline", b"", out.encode(), 0, ctypes.byref(steps))
    assert st == 0, lib.cs_sim_last_error()
    assert os.path.exists(os.path.join(out, "frame3_cloth0.obj"))
    ctx.close()


@pytest.mark.gpu
def test_contact_scene_through_host_layer_matches_c_abi(tmp_path):
    """Two sheets stacked 1.5 mm apart: the host layer detects proximities before every step
    (Simulator::physicsStep, Simulator.cu:571-586) and steps with them; the same sequence through
    the C ABI gives the same frames bit for bit."""
    scene = scenes.stacked_sheets(10, n_layers=2, seed=4)
    path = scenes.write_scene(scene, str(tmp_path / "scene"), frames=1,
                              solver={"tol": 1e-8, "max_iters": 8000, "warm_start": "previous"})
    out = str(tmp_path / "out")
    lib = host()
    steps = ctypes.c_int(0)
    st = lib.cs_sim_run(b"simulate_offline", path.encode(), out.encode(), 0, ctypes.byref(steps))
    assert st == 0, lib.cs_sim_last_error()
    cfg = json.loads(open(path).read().split("\n", 1)[1])  # after the generator's comment line
    n_steps = int(cfg["frame_steps"])
    assert steps.value == n_steps
    ctx = native.Context(0)
    ctx.load(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-8, max_iters=8000,
                           precond_degree=HOST_PRECOND_DEGREE)
    found = []
    for k in range(n_steps):
        p.warm_start = native.WARM_ZERO if k == 0 else native.WARM_PREVIOUS
        found.append(ctx.detect_proximities(1e-3, 1e9, 0.6))
        ctx.step(p)
        ctx.collision_step(scene.dt, COLLISION_THICKNESS)
    assert min(found) > 0
    x, _ = ctx.get_state()
    x = x.reshape(-1, 3)
    o = 0
    for i, s in enumerate(scene.sheets):
        n = s["x"].shape[0]
        xs = [list(map(float, l.split()[1:])) for l in open(os.path.join(out, f"frame1_cloth{i}.obj"))
              if l.startswith("v ")]
        assert np.array_equal(np.array(xs, np.float32), x[o:o + n])
        o += n
    ctx.close()
