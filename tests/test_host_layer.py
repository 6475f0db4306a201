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
    (lambda c: c["handles"][0].__setitem__("motion", 0), "motion index"),
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


def test_host_transformations_and_motions_match_oracle():
    """The host layer's Transformation and Motion (what it hands the C ABI each step) against the
    oracle's FP32 restatement, itself pinned to the reference's classes (test_oracle.py)."""
    import pyoracle
    from test_oracle import MOTION_KEYFRAMES

    lib = host()
    dp = ctypes.POINTER(ctypes.c_double)
    lib.cs_transform_points.argtypes = [ctypes.c_char_p, ctypes.c_int, dp, dp]
    lib.cs_motion_points.argtypes = [ctypes.c_char_p, ctypes.c_int, dp, ctypes.c_int, dp, dp,
                                     ctypes.POINTER(ctypes.c_float)]
    rng = np.random.default_rng(1)
    p = np.ascontiguousarray(rng.normal(size=(30, 3)))
    out = np.zeros_like(p)
    for _ in range(20):
        j = {"scale": float(rng.uniform(0.5, 2)), "translate": rng.normal(size=3).tolist(),
             "rotate": [float(rng.uniform(-180, 180))] + rng.normal(size=3).tolist()}
        assert lib.cs_transform_points(json.dumps(j).encode(), len(p), p.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
        assert np.array_equal(out, pyoracle.transform_points(pyoracle.transform_from_json(j), p).astype(np.float64))
    times = np.arange(1, 90) * 0.01
    out = np.zeros((len(times), len(p), 3))
    tr = np.zeros((len(times), 8), np.float32)
    assert lib.cs_motion_points(json.dumps(MOTION_KEYFRAMES).encode(), len(times), times.ctypes.data_as(dp), len(p),
                                p.ctypes.data_as(dp), out.ctypes.data_as(dp),
                                tr.ctypes.data_as(ctypes.POINTER(ctypes.c_float))) == 0
    m = pyoracle.Motion(MOTION_KEYFRAMES)
    want = [m.transform(t) for t in times]
    assert np.array_equal(tr, np.stack(want))
    assert np.array_equal(out, np.stack([pyoracle.transform_points(w, p) for w in want]).astype(np.float64))


def test_motion_scenes_parse_and_validate(tmp_path):
    from test_oracle import MOTION_KEYFRAMES

    scene = scenes.hang(4, seed=0)
    path = scenes.write_scene(scene, str(tmp_path))
    cfg = json.loads(open(path).read().split("\n", 1)[1])
    cfg["motions"] = [MOTION_KEYFRAMES]
    cfg["handles"][0]["motion"] = 0
    open(path, "w").write(json.dumps(cfg))
    st, counts, err = describe(path)
    assert st == 0, err
    cfg["handles"][0]["motion"] = 1  # no such motion
    open(path, "w").write(json.dumps(cfg))
    st, _, err = describe(path)
    assert st == native.CS_ERR_INVALID_ARG and "motion" in err
    cfg["handles"][0]["motion"] = 0
    cfg["motions"] = {"motfile": "walk.mot", "fps": 30}
    open(path, "w").write(json.dumps(cfg))
    st, _, err = describe(path)
    assert st == native.CS_ERR_INVALID_ARG and ".mot" in err


def read_obj_reference_dialect(path):
    """The reference's OBJ reader restated (Mesh::load, Mesh.cu:306-350, with Mesh::triangulate,
    Mesh.cu:27-54): `v` positions, `nv` velocities, `vt` uv, `f` with a/b (position/uv) or plain
    indices (then a uv from the position's x, y), polygons split as a fan from the corner whose
    fan has the largest smallest angle.  Numbers are read as single precision (std::stof)."""
    x, v, u, fx, fu = [], [], [], [], []

    def angle(a, b, c):
        e1 = (b - a) / np.float32(np.linalg.norm(b - a))
        e2 = (c - a) / np.float32(np.linalg.norm(c - a))
        return float(np.arccos(np.clip(np.float32(np.dot(e1, e2)), -1, 1)))

    for line in open(path):
        s = line.rstrip("\n").split(" ")
        if s[0] == "v":
            x.append(np.array([np.float32(t) for t in s[1:4]], np.float32))
        elif s[0] == "nv":
            v.append(np.array([np.float32(t) for t in s[1:4]], np.float32))
        elif s[0] == "vt":
            u.append(np.array([np.float32(t) for t in s[1:3]], np.float32))
        elif s[0] == "f":
            xp, up = [], []
            for tok in s[1:]:
                if "/" in line:
                    a, b = tok.split("/")[:2]
                    xp.append(int(a) - 1)
                    up.append(int(b) - 1)
                else:
                    xp.append(int(tok) - 1)
                    u.append(x[int(tok) - 1][:2].copy())
                    up.append(len(u) - 1)
            n = len(xp)
            best, index = -np.inf, 0
            for i in range(n):
                m = np.inf
                for j in range(2, n):
                    a, b, c = x[xp[i]], x[xp[(i + j - 1) % n]], x[xp[(i + j) % n]]
                    m = min(m, angle(a, b, c), angle(b, c, a), angle(c, a, b))
                if m > best:
                    best, index = m, i
            for i in range(2, n):
                fx.append([xp[index], xp[(index + i - 1) % n], xp[(index + i) % n]])
                fu.append([up[index], up[(index + i - 1) % n], up[(index + i) % n]])
    v = v + [np.zeros(3, np.float32)] * (len(x) - len(v))
    return (np.array(x, np.float32), np.array(v, np.float32), np.array(u, np.float32), np.array(fx), np.array(fu))


def test_frames_use_the_reference_obj_dialect(tmp_path):
    """A mesh read and written by the host layer (cs_mesh_rewrite: Mesh::load then Mesh::save)
    reads back, through the reference's reader restated, to the same nodes, velocities, uv and
    triangles; every number is written with 20 significant digits (Mesh.cu:456: precision(20)),
    so the single-precision values survive exactly."""
    lib = host()
    lib.cs_mesh_rewrite.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    rng = np.random.default_rng(9)
    s = scenes.grid_sheet(5, rng=rng, z_noise=1e-3, vel_sigma=0.3)
    src = tmp_path / "in.obj"
    scenes.write_obj(s, str(src))
    with open(src, "a") as fh:  # a quad (fan-triangulated) and a face with plain indices
        n = s["x"].shape[0]
        fh.write("v 2 0 0\nnv 0 0 0\nv 3 0 0.1\nnv 0 0 0\nv 3 1 0\nnv 0 0 0\nv 2 1 0.05\nnv 0 0 0\n")
        fh.write("vt 2 0\nvt 3 0\nvt 3 1\nvt 2 1\n")
        nu = s["uv"].shape[0]
        fh.write("f %d/%d %d/%d %d/%d %d/%d\n" % (n + 1, nu + 1, n + 2, nu + 2, n + 3, nu + 3, n + 4, nu + 4))
    out = tmp_path / "out.obj"
    assert lib.cs_mesh_rewrite(str(src).encode(), str(out).encode()) == 0, lib.cs_sim_last_error()
    want = read_obj_reference_dialect(str(src))
    got = read_obj_reference_dialect(str(out))
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    for line in open(out):
        tag, *vals = line.split()
        if tag in ("v", "nv", "vt"):
            for t in vals:
                assert t == "%.20g" % float(np.float32(t)), line
        else:
            assert tag == "f" and len(vals) == 3 and all(len(t.split("/")) == 2 for t in vals)
    plain = tmp_path / "plain.obj"
    plain.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n")
    assert lib.cs_mesh_rewrite(str(plain).encode(), str(out).encode()) == 0
    x, v, u, fx, fu = read_obj_reference_dialect(str(out))
    assert np.array_equal(fx, [[0, 1, 2]]) and np.array_equal(u, [[0, 0], [1, 0], [0, 1]])


def _run(lib, mode, config, directory):
    steps = ctypes.c_int(0)
    rc = lib.cs_sim_run(mode, config.encode() if config else b"", directory.encode(), 0, ctypes.byref(steps))
    assert rc == 0, lib.cs_sim_last_error()


def _frame(directory, frame, cloth):
    return open(os.path.join(directory, f"frame{frame}_cloth{cloth}.obj")).read()


@pytest.mark.gpu
def test_resume_continues_the_trajectory_bit_for_bit(tmp_path):
    """resume_offline from frame 2 (Simulator.cu:936-957, 1070-1083) of two stacked sheets in
    contact falling freely reaches the same frame 3 as a run straight through: the frames hold
    positions and velocities with 20 significant digits (exact single-precision values), and
    every solve starts from the zero guess, so the resumed steps see the state the straight run
    had."""
    scene = scenes.stacked_sheets(8, n_layers=2, seed=6)
    for s in scene.sheets:
        s["handles"] = np.zeros(0, np.int32)
    solver = {"tol": 1e-8, "max_iters": 8000, "warm_start": "zero"}
    lib = host()
    straight, split = str(tmp_path / "straight"), str(tmp_path / "split")
    _run(lib, b"simulate_offline", scenes.write_scene(scene, str(tmp_path / "scene_a"), frames=3, solver=solver), straight)
    _run(lib, b"simulate_offline", scenes.write_scene(scene, str(tmp_path / "scene_b"), frames=2, solver=solver), split)
    assert _frame(straight, 2, 0) == _frame(split, 2, 0)
    cfg = json.load(open(os.path.join(split, "config.json")))
    cfg["end_frame"] = 3
    json.dump(cfg, open(os.path.join(split, "config.json"), "w"))
    _run(lib, b"resume_offline", None, split)
    for i in range(len(scene.sheets)):
        assert _frame(straight, 3, i) == _frame(split, 3, i), f"cloth {i}"


@pytest.mark.gpu
def test_resume_takes_handle_targets_from_the_saved_frame(tmp_path):
    """A resumed simulation is built from the saved config, whose meshes are the last frame's
    OBJ files (Cloth::save, Cloth.cu:865-887), so a fixed handle's target is its node's position
    in that frame (Cloth::addHandles, Cloth.cu:653-664), not the first frame's: resuming from
    frame 2 gives bit for bit the frame a fresh simulate_offline of that saved config reaches
    after one frame, and differs from the straight run's frame 3 (penalty handles sit a little
    off their targets)."""
    scene = scenes.stacked_sheets(8, n_layers=2, seed=6)
    solver = {"tol": 1e-8, "max_iters": 8000, "warm_start": "zero"}
    lib = host()
    straight, split, fresh = str(tmp_path / "straight"), str(tmp_path / "split"), str(tmp_path / "fresh")
    _run(lib, b"simulate_offline", scenes.write_scene(scene, str(tmp_path / "scene_a"), frames=3, solver=solver), straight)
    _run(lib, b"simulate_offline", scenes.write_scene(scene, str(tmp_path / "scene_b"), frames=2, solver=solver), split)
    cfg = json.load(open(os.path.join(split, "config.json")))
    cfg["end_frame"] = 1
    os.makedirs(str(tmp_path / "scene_c"))
    saved = str(tmp_path / "scene_c" / "config.json")
    json.dump(cfg, open(saved, "w"))
    _run(lib, b"simulate_offline", saved, fresh)
    cfg["end_frame"] = 3
    json.dump(cfg, open(os.path.join(split, "config.json"), "w"))
    _run(lib, b"resume_offline", None, split)
    for i in range(len(scene.sheets)):
        assert _frame(split, 3, i) == _frame(fresh, 1, i), f"cloth {i}"
    assert any(_frame(split, 3, i) != _frame(straight, 3, i) for i in range(len(scene.sheets)))
