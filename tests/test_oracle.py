"""The CPU oracle pinned against the reference's own code, and its own consistency checks.

* Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from the reference's
  compiled Material/stretchingForce/bendingForce/Face code) must be reproduced bit for bit by
  the restated FP32 oracle.
* Where the reference adapter is built, it is compared live on more random inputs.
* FP64 oracle: Jacobians against central finite differences where the reference's Jacobian
  is exact (constant stiffness, stretched faces; dihedral angle 0), zero forces at rest, and
  the sparse Cholesky and FP64 PCG against SciPy's direct solve.
"""
import glob
import sys
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import pyoracle
from clothsimulator_b200 import scenes

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_sheet*.npz")))
GOLDEN_PROX = os.path.join(os.path.dirname(__file__), "golden", "ref_prox9.npz")
GOLDEN_DETECT = os.path.join(os.path.dirname(__file__), "golden", "ref_detect.npz")
GOLDEN_COLLIDE = os.path.join(os.path.dirname(__file__), "golden", "ref_collide.npz")


def golden_prox(g):
    mat = {"density": float(g["material_density"]), "stretching": g["material_stretching"].tolist(),
           "bending": g["material_bending"].tolist(), "thicken": 1.0, "density_mult": 1.0,
           "stretching_mult": 1.0, "bending_mult": 1.0}
    sheet = {k: g[k] for k in ("x", "v", "uv", "fx", "fu", "handles")}
    sheet["material"] = mat
    prox = {k[5:]: g[k] for k in g.files if k.startswith("prox_")}
    return sheet, prox


def test_oracle_reproduces_reference_proximity_golden():
    """Repulsion and friction of seeded proximities (the reference's impulseForce and
    frictionForce, PhysicsHelper.cu:398-432), the system assembled with them (Cloth.cu:171-192)
    and one CPU step, bit for bit."""
    g = np.load(GOLDEN_PROX)
    sheet, prox = golden_prox(g)
    c = pyoracle.Cloth(sheet, pyoracle.Material(sheet["material"], "float"))
    c.set_proximities(prox, float(g["thickness"]))
    d, fI, JI, fF, JF = c.proximity_forces(float(g["params"][0]))
    for a, k in [(d, "depth"), (fI, "impulse_f"), (JI, "impulse_J"), (fF, "friction_f"), (JF, "friction_J")]:
        assert np.array_equal(a.astype(np.float32), g[k]), k
    rp, ci, val, b = c.assemble(g["params"])
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col"])
    assert np.array_equal(val.astype(np.float32), g["val"]) and np.array_equal(b.astype(np.float32), g["b"])
    dv, _ = c.step(g["params"], pyoracle.METHOD_LLT)
    x1, v1 = c.state()
    assert np.array_equal(dv.astype(np.float32), g["dv"])
    assert np.array_equal(x1.astype(np.float32), g["x1"]) and np.array_equal(v1.astype(np.float32), g["v1"])


@pytest.mark.ref
def test_oracle_proximities_match_reference_adapter_live():
    if not os.path.exists(pyoracle.LIB_REF):
        pytest.skip("reference adapter not built")
    for seed in range(3):
        rng = np.random.default_rng(100 + seed)
        scene = scenes.uneven_batch(1, seed=seed, nq_range=(6, 12))
        s = scene.sheets[0]
        s["x"] = (s["x"] + rng.normal(0, 0.01, s["x"].shape)).astype(np.float32)
        s["v"] = rng.normal(0, 0.2, s["v"].shape).astype(np.float32)
        prox = scenes.synthetic_proximities(s, rng, n_vf=8, n_ee=6, n_ext=6)
        co = pyoracle.Cloth(s, pyoracle.Material(s["material"]))
        cr = pyoracle.Cloth(s, pyoracle.Material(s["material"], which="ref"))
        for c in (co, cr):
            c.set_proximities(prox, 5e-3)
        for u, w in zip(co.proximity_forces(scene.dt), cr.proximity_forces(scene.dt)):
            assert np.array_equal(u, w)
        p = scenes.step_params(scene, s)
        for u, w in zip(co.assemble(p), cr.assemble(p)):
            assert np.array_equal(u, w)
        d1, _ = co.step(p)
        d2, _ = cr.step(p)
        assert np.array_equal(d1, d2)


def golden_sheet(g):
    mult = g["material_mults"]
    mat = {"density": float(g["material_density"]), "stretching": g["material_stretching"].tolist(),
           "bending": g["material_bending"].tolist(), "thicken": float(mult[0]), "density_mult": float(mult[1]),
           "stretching_mult": float(mult[2]), "bending_mult": float(mult[3])}
    sheet = {k: g[k] for k in ("x", "v", "uv", "fx", "fu", "handles")}
    sheet["material"] = mat
    return sheet, mat


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_reference_golden(path):
    g = np.load(path)
    sheet, mat = golden_sheet(g)
    m = pyoracle.Material(mat, "float")
    assert np.array_equal(m.stretching(g["G"]), g["k"])
    assert np.array_equal(m.bending(g["bend_query"]), g["bend_k"])
    c = pyoracle.Cloth(sheet, m)
    ff, fJ = c.face_forces()
    assert np.array_equal(ff.astype(np.float32), g["face_f"]) and np.array_equal(fJ.astype(np.float32), g["face_J"])
    en, _ = c.interior_edges()
    ef, eJ, th = c.edge_forces()
    assert np.array_equal(en, g["edge_nodes"])
    assert np.array_equal(ef.astype(np.float32), g["edge_f"]) and np.array_equal(eJ.astype(np.float32), g["edge_J"])
    assert np.array_equal(th.astype(np.float32), g["edge_theta"])
    rp, ci, val, b = c.assemble(g["params"])
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col"])
    assert np.array_equal(val.astype(np.float32), g["val"]) and np.array_equal(b.astype(np.float32), g["b"])
    dv, _ = c.step(g["params"], pyoracle.METHOD_LLT)
    x1, v1 = c.state()
    assert np.array_equal(dv.astype(np.float32), g["dv"])
    assert np.array_equal(x1.astype(np.float32), g["x1"]) and np.array_equal(v1.astype(np.float32), g["v1"])


@pytest.mark.ref
def test_oracle_matches_reference_adapter_live():
    if not os.path.exists(pyoracle.LIB_REF):
        pytest.skip("reference adapter not built")
    rng = np.random.default_rng(42)
    for trial in range(3):
        scene = scenes.uneven_batch(1, seed=trial, nq_range=(5, 12))
        s = scene.sheets[0]
        s["x"] = (s["x"] + rng.normal(0, 0.02, s["x"].shape)).astype(np.float32)
        s["v"] = rng.normal(0, 0.2, s["v"].shape).astype(np.float32)
        mo, mr = pyoracle.Material(s["material"]), pyoracle.Material(s["material"], which="ref")
        co, cr = pyoracle.Cloth(s, mo), pyoracle.Cloth(s, mr)
        assert cr.topology_mismatches() == 0
        p = scenes.step_params(scene, s)
        a, b = co.assemble(p), cr.assemble(p)
        for u, w in zip(a, b):
            assert np.array_equal(u, w)
        d1, _ = co.step(p)
        d2, _ = cr.step(p)
        assert np.array_equal(d1, d2)


def _fd_check(sheet, which, eps=1e-6):
    m = pyoracle.Material(sheet["material"], "double")
    c = pyoracle.Cloth(sheet, m)
    x0, v0 = c.state()
    if which == "face":
        f0, J0 = c.face_forces()
        nodes = sheet["fx"]
    else:
        f0, J0, _ = c.edge_forces()
        nodes, _ = c.interior_edges()
    worst = 0.0
    for e in range(min(len(nodes), 6)):
        K = nodes.shape[1]
        Jfd = np.zeros((3 * K, 3 * K))
        for a in range(K):
            for d in range(3):
                xp = x0.copy()
                xm = x0.copy()
                xp[nodes[e, a], d] += eps
                xm[nodes[e, a], d] -= eps
                c.set_state(xp.reshape(-1), v0.reshape(-1))
                fp = (c.face_forces()[0] if which == "face" else c.edge_forces()[0])[e]
                c.set_state(xm.reshape(-1), v0.reshape(-1))
                fm = (c.face_forces()[0] if which == "face" else c.edge_forces()[0])[e]
                Jfd[:, 3 * a + d] = (fp - fm) / (2 * eps)
        c.set_state(x0.reshape(-1), v0.reshape(-1))
        worst = max(worst, np.abs(Jfd - J0[e]).max() / np.abs(J0[e]).max())
    return worst


def test_fp64_stretching_jacobian_matches_finite_differences():
    s = scenes.hang(4, seed=1).sheets[0]
    s["x"] = (s["x"] * np.array([1.05, 1.08, 1.0])).astype(np.float64)  # stretched: G > 0, exact Hessian
    s["x"][:, 2] = 0.0
    assert _fd_check(s, "face") < 1e-6


def test_fp64_bending_jacobian_matches_finite_differences_at_zero_angle():
    s = scenes.hang(4, seed=1).sheets[0]
    s["x"] = s["x"].astype(np.float64)
    s["x"][:, 2] = 0.0  # flat: theta = 0, where the Gauss-Newton Jacobian is exact
    s["x"][:, :2] += np.random.default_rng(0).normal(0, 0.01, (s["x"].shape[0], 2))
    assert _fd_check(s, "edge") < 1e-5


def test_flat_sheet_at_rest_has_no_internal_force():
    s = scenes.hang(6, seed=0).sheets[0]
    s["x"][:, 2] = 0.0
    c = pyoracle.Cloth(s, pyoracle.Material(s["material"], "double"))
    ff, _ = c.face_forces()
    ef, _, th = c.edge_forces()
    assert np.abs(ff).max() < 1e-12 and np.abs(ef).max() < 1e-12 and np.abs(th).max() < 1e-12


def _scipy_system(rp, ci, val, n):
    rows = np.repeat(np.arange(n), np.diff(rp))
    I = (3 * rows[:, None, None] + np.arange(3)[None, :, None]).repeat(3, 2)
    J = (3 * ci[:, None, None] + np.arange(3)[None, None, :]).repeat(3, 1)
    return sp.csr_matrix((val.reshape(-1), (I.reshape(-1), J.reshape(-1))), shape=(3 * n, 3 * n))


def test_sparse_cholesky_and_pcg_match_scipy():
    scene = scenes.hang(10, seed=4)
    s = scene.sheets[0]
    c = pyoracle.Cloth(s, pyoracle.Material(s["material"], "float"))
    rp, ci, val, b = c.assemble(scenes.step_params(scene, s))
    A = _scipy_system(rp, ci, val, c.n)
    ref = spla.spsolve(A.tocsc(), b)
    d64, r64 = c.solve(pyoracle.METHOD_LLT64)
    assert np.linalg.norm(d64 - ref) / np.linalg.norm(ref) < 1e-12 and r64 < 1e-13
    d32, r32 = c.solve(pyoracle.METHOD_LLT)
    assert np.linalg.norm(d32 - ref) / np.linalg.norm(ref) < 1e-3
    dp, rr = c.solve(pyoracle.METHOD_PCG64, tol=1e-13)
    assert np.linalg.norm(dp - ref) / np.linalg.norm(ref) < 1e-9 and rr < 1e-12


def test_topology_counts_for_grid():
    for nq in (1, 2, 5, 16):
        s = scenes.hang(nq, seed=0).sheets[0]
        c = pyoracle.Cloth(s, pyoracle.Material(s["material"]))
        # a grid of nq x nq quads has 3nq^2 + 2nq edges, of which 4nq lie on the boundary
        assert c.L.cloth_num_edges(c.h) == 3 * nq * nq + 2 * nq
        assert c.n_interior == 3 * nq * nq - 2 * nq


def test_oracle_reproduces_reference_detection_golden():
    """Proximity detection over three cloths (a folded sheet, two stacked sheets) as the
    reference's predicates produced it (signedVertexFaceDistance, signedEdgeEdgeDistance,
    inEdge, Proximity constructors): the same proximities, in the same order, bit for bit."""
    g = np.load(GOLDEN_DETECT)
    mat = {"density": float(g["material_density"]), "stretching": g["material_stretching"].tolist(),
           "bending": g["material_bending"].tolist(), "thicken": 1.0, "density_mult": 1.0,
           "stretching_mult": 1.0, "bending_mult": 1.0}
    cloths = []
    for i in range(int(g["n_cloths"])):
        sheet = {k: g[f"c{i}_{k}"] for k in ("x", "v", "uv", "fx", "fu", "handles")}
        cloths.append(pyoracle.Cloth(sheet, pyoracle.Material(mat, "float")))
    det = pyoracle.detect_proximities(cloths, repulsion_thickness=float(g["repulsion_thickness"]),
                                      collision_stiffness=float(g["collision_stiffness"]),
                                      friction=float(g["friction"]))
    assert len(det["mu"]) == len(g["det_mu"]) > 0
    for k, v in det.items():
        ref = g["det_" + k]
        assert np.array_equal(v.astype(ref.dtype), ref), k


@pytest.mark.ref
def test_oracle_detection_matches_reference_adapter_live():
    """The restated detection against the same detection run through the reference's own
    predicates, on self-contact and cross-cloth contact with collision groups."""
    if not os.path.exists(pyoracle.LIB_REF):
        pytest.skip("reference adapter not built")
    cases = [(scenes.folded_sheet(12, seed=1).sheets, None), (scenes.stacked_sheets(10, n_layers=3, seed=2).sheets, None),
             (scenes.stacked_sheets(10, n_layers=3, seed=3).sheets, [0, 0, 1])]
    for sheets, groups in cases:
        out = []
        for which in ("oracle", "ref"):
            cl = [pyoracle.Cloth(s, pyoracle.Material(s["material"], "float", which=which)) for s in sheets]
            out.append(pyoracle.detect_proximities(cl, groups=groups))
        assert len(out[0]["mu"]) > 0
        for k in out[0]:
            assert np.array_equal(out[0][k], out[1][k]), k


def test_oracle_reproduces_reference_collision_golden():
    """Collision steps (impacts, independent selection, impact-zone projection, velocity
    update) as the reference's checkVertexFaceImpact, checkEdgeEdgeImpact and
    CollisionOptimization produced them, on layers driven through each other: rounds and impact
    counts exact; positions within 1e-6 m and velocities within 1e-4 m/s (the reference's
    solveCubic starts Newton's method from an uninitialised value when the derivative is
    degenerate, so the reference itself is reproducible only to Newton's tolerance there; the
    oracle starts from 0)."""
    g = np.load(GOLDEN_COLLIDE)
    mat = {"density": float(g["material_density"]), "stretching": g["material_stretching"].tolist(),
           "bending": g["material_bending"].tolist(), "thicken": 1.0, "density_mult": 1.0,
           "stretching_mult": 1.0, "bending_mult": 1.0}
    for name in ("stacked", "folded"):
        cl = []
        for i in range(int(g[f"{name}_n_cloths"])):
            sheet = {k: g[f"{name}_c{i}_{k}"] for k in ("x", "uv", "fx", "fu", "handles")}
            sheet["v"] = np.zeros_like(sheet["x"])
            c = pyoracle.Cloth(sheet, pyoracle.Material(mat, "float"))
            xe = g[f"{name}_c{i}_xend"]
            c.set_state(xe.astype(np.float64), np.zeros(xe.shape))
            cl.append(c)
        rounds, impacts = pyoracle.collision_step(cl, float(g["dt"]), float(g["thickness"]))
        assert (rounds, impacts) == (int(g[f"{name}_rounds"]), int(g[f"{name}_impacts"])) and impacts > 0, name
        for i, c in enumerate(cl):
            x, v = c.state()
            assert_collided(x, g[f"{name}_c{i}_xout"], name)
            assert_collided(v, g[f"{name}_c{i}_vout"], name, tol=1e-6 / float(g["dt"]))


def assert_collided(a, b, what, tol=1e-6):
    """Within tol: where the reference's solveCubic starts Newton's method from an
    uninitialised value (a degenerate derivative), its own impact times vary from process to
    process by Newton's stopping tolerance; elsewhere the two agree bit for bit."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    assert np.abs(a - b).max() <= tol, what


@pytest.mark.ref
def test_oracle_collision_matches_reference_adapter_live():
    if not os.path.exists(pyoracle.LIB_REF):
        pytest.skip("reference adapter not built")
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden

    for seed in (3, 9):
        for name, scene, xs in make_golden.collide_cases(seed):
            res = []
            for which in ("oracle", "ref"):
                cl = [pyoracle.Cloth(s, pyoracle.Material(s["material"], "float", which=which)) for s in scene.sheets]
                for c, xe in zip(cl, xs):
                    c.set_state(xe.astype(np.float64), np.zeros(xe.shape))
                r = pyoracle.collision_step(cl, 0.01, 1e-4)
                res.append((r, [c.state() for c in cl]))
            assert res[0][0] == res[1][0] and res[0][0][1] > 0, (seed, name)
            for (xa, va), (xb, vb) in zip(res[0][1], res[1][1]):
                assert_collided(xa, xb, (seed, name))
                assert_collided(va, vb, (seed, name), tol=1e-4)


GOLDEN_MATERIALS = os.path.join(os.path.dirname(__file__), "golden", "ref_materials32.npz")


def golden_material_sheets(g):
    """(scene, sheets) of ref_materials32.npz: one 32x32 sheet per reference material file."""
    sheets = []
    for i in range(len(g["names"])):
        p = f"m{i}_"
        par = g[p + "params"]
        mat = {"density": float(g[p + "density"]), "stretching": g[p + "stretching"].tolist(),
               "bending": g[p + "bending"].tolist(), "thicken": 1.0, "density_mult": 1.0, "stretching_mult": 1.0,
               "bending_mult": 1.0}
        s = {"x": g[p + "x"], "v": g[p + "v"], "uv": g["uv"], "fx": g["fx"], "fu": g["fu"], "handles": g["handles"],
             "material": mat, "wind": {"density": float(par[4]), "drag": float(par[5]), "velocity": list(map(float, par[6:9]))}}
        sheets.append(s)
    scene = scenes.Scene("materials", sheets, dt=float(g["m0_params"][0]), steps=1,
                         handle_stiffness=float(g["m0_params"][9]))
    return scene, sheets


def test_oracle_reproduces_reference_material_files():
    """Three of the reference's own material files (gray-interlock, 11oz-black-denim, paper),
    read by the reference's Material: stretching lookups, the windy system's b, the CPU step."""
    g = np.load(GOLDEN_MATERIALS)
    scene, sheets = golden_material_sheets(g)
    for i, s in enumerate(sheets):
        p = f"m{i}_"
        m = pyoracle.Material(s["material"], "float")
        assert m.density == float(g[p + "ref_density"])
        assert np.array_equal(m.stretching(g["G"]), g[p + "k"]), g["names"][i]
        c = pyoracle.Cloth(s, m)
        _, _, _, b = c.assemble(g[p + "params"])
        assert np.array_equal(b.astype(np.float32), g[p + "b"]), g["names"][i]
        dv, _ = c.step(g[p + "params"], pyoracle.METHOD_LLT)
        x1, v1 = c.state()
        assert np.array_equal(dv.astype(np.float32), g[p + "dv"]), g["names"][i]
        assert np.array_equal(x1.astype(np.float32), g[p + "x1"]) and np.array_equal(v1.astype(np.float32), g[p + "v1"])


# Handle motions: Transformation(json).applyToPoint and Motion::computeTransformation, restated in
# FP32 by the oracle, against the reference's own classes (compiled into the adapter).

MOTION_KEYFRAMES = [{"time": 0.1, "transform": {"translate": [0.0, 0.2, 0.1]}},
                    {"time": 0.3, "transform": {"translate": [0.1, 0.3, 0.0], "rotate": [30, 0, 0, 1], "scale": 1.2}},
                    {"time": 0.6, "transform": {"translate": [0.0, 0.0, 0.0], "rotate": [-20, 1, 1, 0]}}]


@pytest.mark.ref
def test_oracle_transformations_and_motions_match_reference():
    if not os.path.exists(pyoracle.LIB_REF):
        pytest.skip("reference adapter not built")
    rng = np.random.default_rng(0)
    p = rng.normal(size=(40, 3))
    for _ in range(30):
        j = {"scale": float(rng.uniform(0.5, 2)), "translate": rng.normal(size=3).tolist(),
             "rotate": [float(rng.uniform(-180, 180))] + rng.normal(size=3).tolist()}
        got = pyoracle.transform_points(pyoracle.transform_from_json(j), p)
        assert np.array_equal(got.astype(np.float64), pyoracle.ref_transform_points(j, p))
    times = np.arange(1, 90) * 0.01  # through every segment and past the last keyframe
    m = pyoracle.Motion(MOTION_KEYFRAMES)
    got = np.stack([pyoracle.transform_points(m.transform(t), p) for t in times])
    assert np.array_equal(got.astype(np.float64), pyoracle.ref_motion_points(MOTION_KEYFRAMES, times, p))
