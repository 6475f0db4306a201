"""Proximity repulsion and friction on the GPU (cs_set_proximities) against the CPU oracle.

The batch mixes sheets with proximities inside them, proximities that couple two sheets
(each sheet gets the terms of its own nodes; the other sheet's nodes enter through their
state, as Cloth::physicsStep sees another cloth's nodes: Cloth.cu:171-192 with index -1),
obstacle-like points outside the batch, and sheets without proximities (solved by the
cluster-resident kernel while the touched ones go to the batched loop).

Tolerances (norm-wise relative):
  * assembled A and b of every touched sheet: 1e-6, pattern identical to the oracle's
    (mesh pattern plus the proximity pairs); the terms are the reference's FP32 arithmetic
    in its accumulation order, so most entries agree bit for bit;
  * dv of a solve to an FP64-checked 1e-10 against an FP64 direct solve of the oracle's
    system: 1e-6;
  * sheets without proximities: bit-identical to a batch without any.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyoracle
from clothsimulator_b200 import native, scenes
from proxutil import offsets, oracle_proximities, touched_sheets

THICKNESS = 5e-3


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))




def face_normal(x, f):
    n = np.cross(x[f[1]] - x[f[0]], x[f[2]] - x[f[0]])
    return n / np.linalg.norm(n)


def cross_sheet(scene, offs, rng, pairs):
    """Vertex-face and edge-edge proximities between sheets a and b (flat sheets at the same
    place: depths of the order of the 1 mm z noise)."""
    recs = {k: [] for k in ("nodes", "x", "v", "mass", "free", "normal", "w", "mu", "stiffness")}
    for a, b in pairs:
        sa, sb = scene.sheets[a], scene.sheets[b]
        xb = sb["x"].astype(np.float64)
        fx = sb["fx"]
        for _ in range(3):
            f = fx[int(rng.integers(len(fx)))]
            i = int(rng.integers(sa["x"].shape[0]))
            bc = rng.dirichlet(np.ones(3))
            recs["nodes"].append([offs[a] + i, *(offs[b] + f)])
            recs["w"].append([1.0, -bc[0], -bc[1], -bc[2]])
            recs["normal"].append(face_normal(xb, f))
            recs["mu"].append(rng.uniform(0.1, 0.6))
            recs["stiffness"].append(rng.uniform(5.0, 40.0))
        for _ in range(2):
            fa = sa["fx"][int(rng.integers(len(sa["fx"])))]
            fb = fx[int(rng.integers(len(fx)))]
            xa = sa["x"].astype(np.float64)
            n = np.cross(xa[fa[1]] - xa[fa[0]], xb[fb[2]] - xb[fb[1]])
            s_, t_ = rng.uniform(0, 1, 2)
            recs["nodes"].append([offs[a] + fa[0], offs[a] + fa[1], offs[b] + fb[1], offs[b] + fb[2]])
            recs["w"].append([1 - s_, s_, -(1 - t_), -t_])
            recs["normal"].append(n / np.linalg.norm(n))
            recs["mu"].append(rng.uniform(0.1, 0.6))
            recs["stiffness"].append(rng.uniform(5.0, 40.0))
    m = len(recs["mu"])
    recs["x"] = np.zeros((m, 4, 3))
    recs["v"] = np.zeros((m, 4, 3))
    recs["mass"] = np.ones((m, 4))
    recs["free"] = np.zeros(m, np.int32)
    return {k: np.asarray(v, dtype=np.int32 if k in ("nodes", "free") else np.float64) for k, v in recs.items()}


def make_case(seed=21, n_sheets=6, nq=12, touched=(0, 1, 2), pairs=((0, 3), (1, 2))):
    scene = scenes.windy_batch(n_sheets, nq, seed=seed)
    rng = np.random.default_rng(seed + 1)
    for s in scene.sheets:  # moving sheets: friction sees tangential velocities
        s["v"] = rng.normal(0, 0.05, s["v"].shape).astype(np.float32)
    offs = offsets(scene)
    parts = [scenes.synthetic_proximities(scene.sheets[k], rng, n_vf=8, n_ee=5, n_ext=4, thickness=THICKNESS,
                                          node_off=int(offs[k])) for k in touched]
    if pairs:
        parts.append(cross_sheet(scene, offs, rng, pairs))
    prox = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    order = rng.permutation(len(prox["mu"]))
    return scene, {k: v[order] for k, v in prox.items()}


def oracle_cloths(scene):
    return [pyoracle.Cloth(s, pyoracle.Material(s["material"], "float")) for s in scene.sheets]






def params_for(scene, **kw):
    kw.setdefault("tol", 1e-10)
    kw.setdefault("max_iters", 20000)
    return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, **kw)


def gpu_sheet_system(sys, offs, k):
    rp, ci, val, b = sys
    lo, hi = offs[k], offs[k + 1]
    r = rp[lo:hi + 1] - rp[lo]
    c = ci[rp[lo]:rp[hi]] - lo
    assert c.min() >= 0 and c.max() < hi - lo, "a block couples two sheets"
    return r, c, val[rp[lo]:rp[hi]], b[3 * lo:3 * hi]


def set_oracle_proximities(cloths, scene, prox, offs):
    x = np.concatenate([s["x"] for s in scene.sheets]).astype(np.float64)
    v = np.concatenate([s["v"] for s in scene.sheets]).astype(np.float64)
    mass = np.concatenate([c.masses() for c in cloths])
    for k in touched_sheets(prox, offs):
        cloths[k].set_proximities(oracle_proximities(prox, k, offs, x, v, mass), THICKNESS)


def mesh_pattern(sheet):
    c = pyoracle.Cloth(sheet, pyoracle.Material(sheet["material"], "float"))
    rp, ci, _, _ = c.assemble([1e-2, 0, 0, 0, 0, 0, 0, 0, 0, 0])
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    return set(zip(rows.tolist(), ci.tolist()))


def test_proximity_system_matches_oracle(ctx_factory):
    scene, prox = make_case()
    offs = offsets(scene)
    ctx = ctx_factory(scene.sheets)
    nnzb0 = ctx.sizes[6]
    ctx.set_proximities(prox, THICKNESS)
    assert ctx.sizes[6] > nnzb0, "the case should have proximity blocks outside the mesh pattern"
    ctx.assemble(params_for(scene))
    sys = ctx.system()
    cloths = oracle_cloths(scene)
    set_oracle_proximities(cloths, scene, prox, offs)
    touched = touched_sheets(prox, offs)
    assert touched == [0, 1, 2, 3]
    n_outside = 0
    for k in range(len(scene.sheets)):
        rp, ci, val, b = gpu_sheet_system(sys, offs, k)
        orp, oci, oval, ob = cloths[k].assemble(scenes.step_params(scene, scene.sheets[k]))
        assert np.array_equal(rp, orp) and np.array_equal(ci, oci), f"sheet {k}: pattern differs"
        assert rel(val, oval) < 1e-6 and rel(b, ob) < 1e-6, f"sheet {k}"
        # blocks outside the mesh pattern hold proximity terms only: bit for bit
        mesh = mesh_pattern(scene.sheets[k])
        rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
        outside = np.array([(i, j) not in mesh for i, j in zip(rows, ci)], bool)
        n_outside += int(outside.sum())
        ov = oval.astype(np.float32)
        assert np.array_equal(val[outside], ov[outside]), f"sheet {k}: proximity-only blocks differ"
        # the mesh terms' transcendentals (host libm vs CUDA) leave a few ulps in ~1 % of entries
        assert np.mean(val == ov) > 0.98 and np.mean(b == ob.astype(np.float32)) > 0.98, f"sheet {k}"
    assert n_outside > 0


def test_proximity_solve_matches_fp64_oracle(ctx_factory):
    scene, prox = make_case(seed=22)
    offs = offsets(scene)
    ref = ctx_factory(scene.sheets)
    ctx = ctx_factory(scene.sheets)
    full = ctx.solver_info()["resident_sheets"]
    ctx.set_proximities(prox, THICKNESS)
    touched = touched_sheets(prox, offs)
    if full:
        assert ctx.solver_info()["resident_sheets"] == full - len(touched)
    stats, _ = ctx.step(params_for(scene, advance=0))
    assert stats.converged == len(scene.sheets) and stats.max_rel_residual <= 1e-10
    dv = ctx.get_dv().reshape(-1)
    stats0, _ = ref.step(params_for(scene, advance=0))
    dv0 = ref.get_dv().reshape(-1)
    cloths = oracle_cloths(scene)
    set_oracle_proximities(cloths, scene, prox, offs)
    for k in range(len(scene.sheets)):
        lo, hi = 3 * offs[k], 3 * offs[k + 1]
        if k in touched:
            cloths[k].assemble(scenes.step_params(scene, scene.sheets[k]))
            odv, _ = cloths[k].solve(pyoracle.METHOD_LLT64)
            assert rel(dv[lo:hi], odv) < 1e-6, f"sheet {k}"
            assert rel(dv[lo:hi], dv0[lo:hi]) > 1e-4, f"sheet {k}: proximities had no effect"
        else:
            assert np.array_equal(dv[lo:hi], dv0[lo:hi]), f"sheet {k}: untouched sheet changed"


@pytest.mark.parametrize("solver,use_graph", [(native.SOLVER_BATCHED, 1), (native.SOLVER_AUTO, 0)])
def test_proximity_solver_paths_agree(ctx_factory, solver, use_graph):
    scene, prox = make_case(seed=23)
    a = ctx_factory(scene.sheets)
    b = ctx_factory(scene.sheets)
    for c in (a, b):
        c.set_proximities(prox, THICKNESS)
    a.step(params_for(scene, advance=0))
    b.step(params_for(scene, advance=0, solver=solver, use_graph=use_graph))
    assert rel(b.get_dv(), a.get_dv()) < 1e-6


def test_proximity_steps_track_oracle(ctx_factory):
    """Three steps with the proximities held: every sheet against the oracle stepping the
    same cloths, the outside points of each step taken from the oracle's states."""
    scene, prox = make_case(seed=24)
    offs = offsets(scene)
    ctx = ctx_factory(scene.sheets)
    ctx.set_proximities(prox, THICKNESS)
    cloths = oracle_cloths(scene)
    mass = np.concatenate([c.masses() for c in cloths])
    for _ in range(3):
        xs = np.concatenate([c.state()[0] for c in cloths])
        vs = np.concatenate([c.state()[1] for c in cloths])
        for k in touched_sheets(prox, offs):
            cloths[k].set_proximities(oracle_proximities(prox, k, offs, xs, vs, mass), THICKNESS)
        for k, c in enumerate(cloths):
            c.step(scenes.step_params(scene, scene.sheets[k]), pyoracle.METHOD_LLT64)
        stats, _ = ctx.step(params_for(scene))
        assert stats.converged == len(scene.sheets)
    x, _ = ctx.get_state()
    x = x.reshape(-1, 3)
    x0 = np.concatenate([s["x"] for s in scene.sheets]).astype(np.float64)
    xo = np.concatenate([c.state()[0] for c in cloths])
    assert rel(x - x0, xo - x0) < 1e-5


def test_clearing_proximities_restores_the_batch(ctx_factory):
    scene, prox = make_case(seed=25)
    ctx = ctx_factory(scene.sheets)
    info0, nnzb0 = ctx.solver_info(), ctx.sizes[6]
    ctx.assemble(params_for(scene))
    sys0 = ctx.system()
    ctx.set_proximities(prox, THICKNESS)
    ctx.step(params_for(scene, advance=0))
    ctx.set_proximities(None)
    assert ctx.solver_info() == info0 and ctx.sizes[6] == nnzb0
    ctx.assemble(params_for(scene))
    for u, w in zip(sys0, ctx.system()):
        assert np.array_equal(u, w)


def test_proximity_arguments_are_checked(ctx_factory):
    scene, prox = make_case(seed=26, n_sheets=2, touched=(0,), pairs=())
    ctx = ctx_factory(scene.sheets)
    bad = {k: v.copy() for k, v in prox.items()}
    bad["nodes"][0, 1] = ctx.n  # past the batch
    with pytest.raises(native.ClothStepError):
        ctx.set_proximities(bad, THICKNESS)
    with pytest.raises(native.ClothStepError):
        ctx.set_proximities(prox, 0.0)
    bad = {k: v.copy() for k, v in prox.items()}
    ext = int(np.argmax((bad["nodes"] < 0).any(axis=1)))
    assert (bad["nodes"][ext] < 0).any()
    bad["free"][ext] = 1
    bad["mass"][ext, 0] = 0.0  # a free outside point needs a mass
    with pytest.raises(native.ClothStepError):
        ctx.set_proximities(bad, THICKNESS)
    # a rejected call leaves the batch as it was
    assert ctx.sizes[6] == ctx.get_sizes()[6]
    stats, _ = ctx.step(params_for(scene, advance=0))
    assert stats.converged == len(scene.sheets)
