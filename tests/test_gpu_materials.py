"""GPU parity on data-driven materials: anisotropic stretching tables and varied bending samples.

The other GPU tests mostly use isotropic rows [E, 0, E, E] and constant bending samples, under
which a wrong index, weight or clamp in the trilinear stretching lookup or the bilinear bending
lookup (Material.cu:91-156) would not show.  Here:

  * tests/golden/ref_sheet6.npz, ref_sheet9.npz: seeded anisotropic materials with thicken and
    stretching/bending multipliers, run through the reference's own Material, stretchingForce
    and bendingForce (PhysicsHelper.cu:264-353) and its CPU step (FP32 sparse LL^T);
  * tests/golden/ref_materials32.npz: three of the reference's own material files
    (gray-interlock, 11oz-black-denim, paper; Material.cu:3-41 reads them) on windy 32x32 sheets,
    loaded as one batch with three materials, so the system also carries the wind forces.

Bars (norm-wise relative): element forces and Jacobians 1e-6 with > 99 % of the face entries bit
for bit; assembled A and b 1e-6; dv of a solve to an FP64-checked relative residual of 1e-10
against the reference's FP32 LL^T within 1e-5, or 1.5x that LL^T's own error against an FP64
solve of the same system when it is larger, and against the FP64 solve within 1e-6.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyoracle
from clothsimulator_b200 import native, scenes

from test_oracle import golden_material_sheets, golden_sheet

HERE = os.path.dirname(__file__)
GOLDEN_SHEETS = [os.path.join(HERE, "golden", f) for f in ("ref_sheet6.npz", "ref_sheet9.npz")]
GOLDEN_MATERIALS = os.path.join(HERE, "golden", "ref_materials32.npz")


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def params_from(packed, **kw):
    """Step parameters of a packed [dt, g(3), wind density, drag, wind velocity(3), k_handle]."""
    kw.setdefault("tol", 1e-10)
    kw.setdefault("max_iters", 40000)
    return native.step_params(float(packed[0]), tuple(float(v) for v in packed[1:4]), float(packed[9]), **kw)


def fp64_solve(sheet, packed):
    oc = pyoracle.Cloth(sheet, pyoracle.Material(sheet["material"], "float"))
    oc.assemble(packed)
    ref, _ = oc.solve(pyoracle.METHOD_LLT64)
    return ref


@pytest.mark.parametrize("path", GOLDEN_SHEETS, ids=[os.path.basename(p) for p in GOLDEN_SHEETS])
def test_anisotropic_golden_sheet(ctx_factory, path):
    g = np.load(path)
    sheet, _ = golden_sheet(g)
    packed = g["params"]
    sheet["wind"] = {"density": float(packed[4]), "drag": float(packed[5]), "velocity": list(map(float, packed[6:9]))}
    ctx = ctx_factory([sheet])
    p = params_from(packed, advance=0)
    ctx.assemble(p)
    ff, fJ, ef, eJ, en = ctx.element_forces()
    assert np.array_equal(en, g["edge_nodes"])
    assert rel(ff, g["face_f"]) < 1e-6 and rel(fJ, g["face_J"]) < 1e-6
    assert rel(ef, g["edge_f"]) < 1e-6 and rel(eJ, g["edge_J"]) < 1e-6
    assert np.mean(ff == g["face_f"]) > 0.99 and np.mean(fJ == g["face_J"]) > 0.99
    rp, ci, val, b = ctx.system()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col"])
    assert rel(val, g["val"]) < 1e-6 and rel(b, g["b"]) < 1e-6
    stats, _ = ctx.step(p)
    assert stats.converged == 1 and stats.max_rel_residual <= 1e-10
    dv = ctx.get_dv().reshape(-1)
    exact = fp64_solve(sheet, packed)
    ref_err = rel(g["dv"], exact)
    assert rel(dv, exact) < 1e-6
    assert rel(dv, g["dv"]) < max(1e-5, 1.5 * ref_err), f"reference FP32 LL^T error {ref_err:.2e}"


def test_reference_material_files_batch(ctx_factory):
    g = np.load(GOLDEN_MATERIALS)
    scene, sheets = golden_material_sheets(g)
    ctx = ctx_factory(sheets)
    packed = [g[f"m{i}_params"] for i in range(len(sheets))]
    p = params_from(packed[0], advance=0)
    ctx.assemble(p)
    ff, fJ, ef, eJ, en = ctx.element_forces()
    rp, ci, val, b = ctx.system()
    nf, n = sheets[0]["fx"].shape[0], sheets[0]["x"].shape[0]
    ne = en.shape[0] // len(sheets)
    for i, s in enumerate(sheets):
        name = str(g["names"][i])
        oc = pyoracle.Cloth(s, pyoracle.Material(s["material"], "float"))
        of, oJ = oc.face_forces()
        oef, oeJ, _ = oc.edge_forces()
        sf, se, sn = slice(i * nf, (i + 1) * nf), slice(i * ne, (i + 1) * ne), slice(3 * i * n, 3 * (i + 1) * n)
        assert rel(ff[sf], of) < 1e-6 and rel(fJ[sf], oJ) < 1e-6, name
        assert np.mean(ff[sf] == of.astype(np.float32)) > 0.99 and np.mean(fJ[sf] == oJ.astype(np.float32)) > 0.99, name
        assert rel(ef[se], oef) < 1e-6 and rel(eJ[se], oeJ) < 1e-6, name
        orp, oci, oval, ob = oc.assemble(packed[i])
        blocks = slice(rp[i * n], rp[(i + 1) * n])
        assert np.array_equal(rp[i * n:(i + 1) * n + 1] - rp[i * n], orp), name
        assert np.array_equal(ci[blocks] - i * n, oci), name
        assert rel(val[blocks], oval) < 1e-6, name
        # b against the reference's own assembly (wind, gravity, handles, internal forces)
        assert rel(b[sn], g[f"m{i}_b"]) < 1e-6, name
    stats, _ = ctx.step(p)
    assert stats.converged == len(sheets) and stats.max_rel_residual <= 1e-10
    dv = ctx.get_dv().reshape(-1)
    for i, s in enumerate(sheets):
        name = str(g["names"][i])
        sn = slice(3 * i * n, 3 * (i + 1) * n)
        exact = fp64_solve(s, packed[i])
        ref_err = rel(g[f"m{i}_dv"], exact)
        assert rel(dv[sn], exact) < 1e-6, name
        assert rel(dv[sn], g[f"m{i}_dv"]) < max(1e-5, 1.5 * ref_err), f"{name}: reference LL^T error {ref_err:.2e}"


def test_reference_material_files_step_positions(ctx_factory):
    """A full step (v += dv, x += dt v) of the three material sheets against the reference CPU
    path's state after its step: v - v0 within the dv bar; x differs from the reference's by no
    more than dt times the difference of the velocities plus one FP32 rounding of x (the
    reference's FP32 LL^T carries its own error into both, largest for the stiff paper)."""
    g = np.load(GOLDEN_MATERIALS)
    scene, sheets = golden_material_sheets(g)
    ctx = ctx_factory(sheets)
    stats, _ = ctx.step(params_from(g["m0_params"], advance=1))
    assert stats.converged == len(sheets)
    x, v = ctx.get_state()
    n = sheets[0]["x"].shape[0]
    for i, s in enumerate(sheets):
        name = str(g["names"][i])
        xi, vi = x[i * n:(i + 1) * n], v[i * n:(i + 1) * n]
        dt = float(g[f"m{i}_params"][0])
        dvel = np.linalg.norm(vi.astype(np.float64) - g[f"m{i}_v1"])
        assert np.linalg.norm(xi.astype(np.float64) - g[f"m{i}_x1"]) <= 1.01 * dt * dvel + 1.2e-7 * np.sqrt(xi.size), name
        exact = fp64_solve(s, g[f"m{i}_params"])
        ref_err = rel(g[f"m{i}_dv"], exact)
        assert rel(vi - s["v"], g[f"m{i}_v1"] - s["v"]) < max(1e-5, 1.5 * ref_err) + 1e-6, name
