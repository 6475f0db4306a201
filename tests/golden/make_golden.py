"""Generates tests/golden/*.npz from the reference's own code.

Run in a checkout where the reference adapter (oracle/_ref/libclothref.so, built by
``make -C oracle ref`` from the reference sources) exists:

    python tests/golden/make_golden.py

The fixtures hold inputs and the outputs of the reference's Material, stretchingForce,
bendingForce and Face code (PhysicsHelper.cu:264-353, Material.cu:3-156, Face.cu:12-20,
124-132), the system assembled around them in the reference order (Cloth.cu:42-169) and
one CPU-path step (FP32 sparse Cholesky).  Materials are seeded synthetic parameter sets
(anisotropic stretching rows, varied bending samples), not the reference's material files.
ref_prox9.npz adds seeded proximities: the reference's impulseForce and frictionForce per
proximity and the step with them (`python tests/golden/make_golden.py ref_prox9` makes only
that file).  ref_detect.npz holds proximity detection over three cloths (a sheet folded over
itself, two stacked sheets) through the reference's own signedVertexFaceDistance,
signedEdgeEdgeDistance, inEdge and Proximity constructors (MathHelper.cu:38-69,
PhysicsHelper.cu:3-18, Proximity.cu:5-21).  ref_collide.npz holds collision steps
(Simulator::collisionStep) through the reference's own checkVertexFaceImpact,
checkEdgeEdgeImpact and CollisionOptimization: two stacked sheets and a folded sheet whose upper
layers were driven through the lower ones during the step.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from clothsimulator_b200 import scenes  # noqa: E402


def synthetic_material(rng):
    rows = []
    for _ in range(6):
        a = rng.uniform(10, 300)
        rows.append([a, rng.uniform(-0.5, 0.5) * a, rng.uniform(0.5, 2.0) * a, rng.uniform(-0.3, 0.3) * a])
    bend = rng.uniform(5e-6, 5e-5, size=(3, 5))
    return {"density": float(rng.uniform(0.1, 0.4)), "stretching": [list(map(float, r)) for r in rows],
            "bending": bend.tolist(), "thicken": 2.0, "density_mult": 1.0, "stretching_mult": 1.5,
            "bending_mult": 0.5}


def make_case(seed, nq, amp):
    rng = np.random.default_rng(seed)
    mat = synthetic_material(rng)
    scene = scenes.hang(nq, seed=seed)
    s = scene.sheets[0]
    s["material"] = mat
    s["x"] = (s["x"] + rng.normal(0, amp, s["x"].shape)).astype(np.float32)
    s["v"] = rng.normal(0, 0.1, s["v"].shape).astype(np.float32)
    m = pyoracle.Material(mat, which="ref")
    G = np.column_stack([rng.uniform(-0.3, 1.0, 400), rng.uniform(-0.6, 0.6, 400), rng.uniform(-0.3, 1.0, 400)])
    q = np.column_stack([rng.uniform(0.01, 0.2, 400), rng.uniform(-3, 3, 400), rng.uniform(1e-4, 1e-2, 400),
                         rng.normal(0, 1, 400), rng.normal(0, 1, 400)])
    c = pyoracle.Cloth(s, m)
    assert c.topology_mismatches() == 0
    ff, fJ = c.face_forces()
    ef, eJ, th = c.edge_forces()
    en, efaces = c.interior_edges()
    params = np.array(scenes.step_params(scene, s))
    rp, ci, val, b = c.assemble(params)
    dv, rr = c.step(params, pyoracle.METHOD_LLT)
    x1, v1 = c.state()
    return dict(
        material_density=mat["density"], material_stretching=np.array(mat["stretching"]),
        material_bending=np.array(mat["bending"]), material_mults=np.array([2.0, 1.0, 1.5, 0.5]),
        G=G, k=m.stretching(G), bend_query=q, bend_k=m.bending(q),
        x=s["x"], v=s["v"], uv=s["uv"], fx=s["fx"], fu=s["fu"], handles=s["handles"], params=params,
        face_f=ff.astype(np.float32), face_J=fJ.astype(np.float32), edge_nodes=en,
        edge_f=ef.astype(np.float32), edge_J=eJ.astype(np.float32), edge_theta=th.astype(np.float32),
        row_ptr=rp, col=ci, val=val.astype(np.float32), b=b.astype(np.float32),
        dv=dv.astype(np.float32), x1=x1.astype(np.float32), v1=v1.astype(np.float32),
    )


REFERENCE_MATERIALS = ("gray-interlock", "11oz-black-denim", "paper")


def read_material_file(path):
    """Density, stretching rows and bending samples of a material data file in the reference's
    format (materials/*.json; `//` comment lines allowed, as the reference's reader takes them)."""
    import json

    text = "\n".join(line for line in open(path).read().splitlines() if not line.lstrip().startswith("//"))
    d = json.loads(text)
    return {"density": float(d["density"]), "stretching": [[float(v) for v in r] for r in d["stretching"]],
            "bending": [[float(v) for v in r] for r in d["bending"]]}


def make_materials_case(materials_dir, nq=32, seed=51):
    """A 32x32 sheet, top edge pinned, per-material wind, perturbed state, run through each of
    three of the reference's own material files (Material.cu:3-41 reads the file itself here):
    the reference's stretching lookups at seeded strains, and per material the right-hand side
    b of the system assembled in the reference order (Cloth.cu:78-169, wind included), the
    CPU-path step's dv (FP32 sparse LL^T) and the state after it."""
    rng = np.random.default_rng(seed)
    base = scenes.grid_sheet(nq, rng=rng, z_noise=1e-3)
    out = {"names": np.array(REFERENCE_MATERIALS), "uv": base["uv"], "fx": base["fx"], "fu": base["fu"],
           "handles": scenes.top_edge(nq)}
    G = np.column_stack([rng.uniform(-0.3, 1.0, 400), rng.uniform(-0.6, 0.6, 400), rng.uniform(-0.3, 1.0, 400)])
    out["G"] = G
    for i, name in enumerate(REFERENCE_MATERIALS):
        path = os.path.join(materials_dir, name + ".json")
        mat = read_material_file(path)
        mat.update({"thicken": 1.0, "density_mult": 1.0, "stretching_mult": 1.0, "bending_mult": 1.0})
        s = {k: base[k] for k in ("uv", "fx", "fu")}
        s["handles"] = out["handles"]
        s["x"] = (base["x"] + rng.normal(0, 4e-3, base["x"].shape)).astype(np.float32)
        s["v"] = rng.normal(0, 0.05, base["x"].shape).astype(np.float32)
        phi = rng.uniform(0.0, 2.0 * np.pi)
        speed = rng.uniform(2.0, 8.0)
        s["wind"] = {"density": 1.0, "drag": 1.0, "velocity": [speed * np.cos(phi), 0.0, speed * np.sin(phi)]}
        s["material"] = mat
        scene = scenes.Scene("materials", [s], dt=1.0 / 100, steps=1)
        m = pyoracle.Material(dict(mat, data_file=path), which="ref")
        c = pyoracle.Cloth(s, m)
        assert c.topology_mismatches() == 0
        params = np.array(scenes.step_params(scene, s))
        _, _, _, b = c.assemble(params)
        dv, _ = c.step(params, pyoracle.METHOD_LLT)
        x1, v1 = c.state()
        p = f"m{i}_"
        out.update({p + "density": mat["density"], p + "stretching": np.array(mat["stretching"]),
                    p + "bending": np.array(mat["bending"]), p + "ref_density": m.density,
                    p + "k": m.stretching(G), p + "x": s["x"], p + "v": s["v"], p + "params": params,
                    p + "b": b.astype(np.float32), p + "dv": dv.astype(np.float32), p + "x1": x1.astype(np.float32),
                    p + "v1": v1.astype(np.float32)})
    return out


THICKNESS = 5e-3


def make_prox_case(seed, nq):
    """A hanging sheet with seeded proximities (vertex-face, edge-edge, external points): the
    reference's impulseForce and frictionForce (PhysicsHelper.cu:398-432) per proximity, the
    system assembled with them in the reference order (Cloth.cu:171-192) and one CPU step."""
    rng = np.random.default_rng(seed)
    scene = scenes.hang(nq, seed=seed)
    s = scene.sheets[0]
    s["x"] = (s["x"] + rng.normal(0, 0.01, s["x"].shape)).astype(np.float32)
    s["v"] = rng.normal(0, 0.1, s["v"].shape).astype(np.float32)
    prox = scenes.synthetic_proximities(s, rng, thickness=THICKNESS)
    c = pyoracle.Cloth(s, pyoracle.Material(s["material"], which="ref"))
    c.set_proximities(prox, THICKNESS)
    params = np.array(scenes.step_params(scene, s))
    d, fI, JI, fF, JF = c.proximity_forces(scene.dt)
    rp, ci, val, b = c.assemble(params)
    dv, _ = c.step(params, pyoracle.METHOD_LLT)
    x1, v1 = c.state()
    out = dict(x=s["x"], v=s["v"], uv=s["uv"], fx=s["fx"], fu=s["fu"], handles=s["handles"], params=params,
               thickness=THICKNESS, depth=d.astype(np.float32), impulse_f=fI.astype(np.float32),
               impulse_J=JI.astype(np.float32), friction_f=fF.astype(np.float32), friction_J=JF.astype(np.float32),
               row_ptr=rp, col=ci, val=val.astype(np.float32), b=b.astype(np.float32), dv=dv.astype(np.float32),
               x1=x1.astype(np.float32), v1=v1.astype(np.float32))
    out.update({"prox_" + k: v for k, v in prox.items()})
    out["material_stretching"] = np.array(s["material"]["stretching"])
    out["material_bending"] = np.array(s["material"]["bending"])
    out["material_density"] = s["material"]["density"]
    return out


def make_detect_case(seed):
    """Proximities among a folded sheet (moved 2 m along x, apart from the others) and two
    stacked sheets, detected through the reference's predicates (Simulator.cu:198-298)."""
    folded = scenes.folded_sheet(8, seed=seed).sheets[0]
    folded["x"] = (folded["x"] + np.array([2.0, 0.0, 0.0], np.float32)).astype(np.float32)
    cloths = [folded] + scenes.stacked_sheets(8, n_layers=2, seed=seed + 1).sheets
    refs = [pyoracle.Cloth(c, pyoracle.Material(c["material"], which="ref")) for c in cloths]
    det = pyoracle.detect_proximities(refs, repulsion_thickness=1e-3)
    out = {"n_cloths": len(cloths), "repulsion_thickness": 1e-3, "collision_stiffness": 1e9, "friction": 0.6}
    for i, c in enumerate(cloths):
        for k in ("x", "v", "uv", "fx", "fu", "handles"):
            out[f"c{i}_{k}"] = c[k]
    m = cloths[0]["material"]
    out["material_stretching"] = np.array(m["stretching"])
    out["material_bending"] = np.array(m["bending"])
    out["material_density"] = m["density"]
    for k, v in det.items():
        out["det_" + k] = v.astype(np.float32) if v.dtype == np.float64 else v
    return out


def collide_cases(seed):
    """(name, scene, end positions per cloth): layers driven through each other in a step."""
    stacked = scenes.stacked_sheets(8, n_layers=2, seed=seed)
    xs = [s["x"].astype(np.float32).copy() for s in stacked.sheets]
    xs[1][:, 2] -= np.float32(3e-3)
    folded = scenes.folded_sheet(10, seed=seed + 1)
    xf = folded.sheets[0]["x"].astype(np.float32).copy()
    up = xf[:, 2] > 0.75e-3
    xf[up, 2] -= np.float32(3.75e-3)
    return [("stacked", stacked, xs), ("folded", folded, [xf])]


def make_collide_case(seed):
    out = {"dt": 0.01, "thickness": 1e-4}
    m = None
    for name, scene, xs in collide_cases(seed):
        cl = [pyoracle.Cloth(s, pyoracle.Material(s["material"], which="ref")) for s in scene.sheets]
        for c, xe in zip(cl, xs):
            c.set_state(xe.astype(np.float64), np.zeros(xe.shape))
        rounds, impacts = pyoracle.collision_step(cl, 0.01, 1e-4)
        out[f"{name}_n_cloths"] = len(scene.sheets)
        for i, (s, xe, c) in enumerate(zip(scene.sheets, xs, cl)):
            for k in ("x", "uv", "fx", "fu", "handles"):
                out[f"{name}_c{i}_{k}"] = s[k]
            out[f"{name}_c{i}_xend"] = xe
            x, v = c.state()
            out[f"{name}_c{i}_xout"] = x.astype(np.float32)
            out[f"{name}_c{i}_vout"] = v.astype(np.float32)
        out[f"{name}_rounds"] = rounds
        out[f"{name}_impacts"] = impacts
        m = scene.sheets[0]["material"]
    out["material_stretching"] = np.array(m["stretching"])
    out["material_bending"] = np.array(m["bending"])
    out["material_density"] = m["density"]
    return out


if __name__ == "__main__":
    only = sys.argv[1:]
    for name, seed, nq, amp in [("ref_sheet6", 11, 6, 0.03), ("ref_sheet9", 12, 9, 0.01)]:
        if only and name not in only:
            continue
        case = make_case(seed, nq, amp)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **case)
        print(name, {k: np.asarray(v).shape for k, v in case.items() if np.asarray(v).size > 1})
    if not only or "ref_prox9" in only:
        case = make_prox_case(21, 9)
        np.savez_compressed(os.path.join(HERE, "ref_prox9.npz"), **case)
        print("ref_prox9", {k: np.asarray(v).shape for k, v in case.items() if np.asarray(v).size > 1})
    if not only or "ref_collide" in only:
        case = make_collide_case(41)
        np.savez_compressed(os.path.join(HERE, "ref_collide.npz"), **case)
        print("ref_collide", {k: int(v) for k, v in case.items() if k.endswith(("rounds", "impacts"))})
    if not only or "ref_materials32" in only:
        # the reference checkout's materials directory: REFERENCE_MATERIALS_DIR, else next to
        # the sources the oracle's adapter was built from
        mdir = os.environ.get("REFERENCE_MATERIALS_DIR") or os.path.join(
            os.path.dirname(pyoracle.reference_src()), "materials")
        case = make_materials_case(mdir)
        np.savez_compressed(os.path.join(HERE, "ref_materials32.npz"), **case)
        print("ref_materials32", [str(n) for n in case["names"]])
    if not only or "ref_detect" in only:
        case = make_detect_case(31)
        np.savez_compressed(os.path.join(HERE, "ref_detect.npz"), **case)
        print("ref_detect", {k: np.asarray(v).shape for k, v in case.items() if k.startswith("det_")})
