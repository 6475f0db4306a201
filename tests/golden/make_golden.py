"""Generates tests/golden/*.npz from the reference's own code.

Run in a checkout where the reference adapter (oracle/_ref/libclothref.so, built by
``make -C oracle ref`` from the reference sources) exists:

    python tests/golden/make_golden.py

The fixtures hold inputs and the outputs of the reference's Material, stretchingForce,
bendingForce and Face code (PhysicsHelper.cu:264-353, Material.cu:3-156, Face.cu:12-20,
124-132), the system assembled around them in the reference order (Cloth.cu:42-169) and
one CPU-path step (FP32 sparse Cholesky).  Materials are seeded synthetic parameter sets
(anisotropic stretching rows, varied bending samples), not the reference's material files.
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


if __name__ == "__main__":
    for name, seed, nq, amp in [("ref_sheet6", 11, 6, 0.03), ("ref_sheet9", 12, 9, 0.01)]:
        case = make_case(seed, nq, amp)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **case)
        print(name, {k: np.asarray(v).shape for k, v in case.items() if np.asarray(v).size > 1})
