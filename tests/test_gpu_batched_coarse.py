"""The batched loop's coarse-space correction (coarse.cu): aggregates of about 256 nodes binned
by rest (u, v), the additive two-level preconditioner D^-1 + R^T A_c^-1 R with A_c = R A R^T
inverted per step (one CTA up to 192 coarse unknowns, a 16-CTA cluster above).

Bars (norm-wise relative): dv of a solve to an FP64-checked relative residual of 1e-10
against an FP64 direct solve of the same system (SciPy) within 1e-6, as for the loop without
the correction; fewer CG iterations than block-Jacobi alone (the point of the correction);
bit-for-bit repeatability; the correction off (coarse = 0) leaves the loop as it was."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spl

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native, scenes


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def params(scene, **kw):
    kw.setdefault("tol", 1e-10)
    kw.setdefault("max_iters", 40000)
    kw.setdefault("advance", 0)
    return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, solver=native.SOLVER_BATCHED, **kw)


def fp64_dv(ctx, p, ranges):
    """Per sheet, the FP64 direct solve of the system the GPU assembled."""
    ctx.assemble(p)
    rp, ci, val, b = ctx.system()
    n = rp.shape[0] - 1
    A = sp.bsr_matrix((val.astype(np.float64), ci, rp), shape=(3 * n, 3 * n)).tocsc()
    out = []
    for n0, n1 in ranges:
        sl = slice(3 * n0, 3 * n1)
        out.append(spl.spsolve(A[sl, sl], b.astype(np.float64)[sl]))
    return out


def ranges_of(scene):
    r, off = [], 0
    for s in scene.sheets:
        r.append((off, off + s["x"].shape[0]))
        off += s["x"].shape[0]
    return r


@pytest.mark.parametrize("nq,path", [(96, "one CTA (108 coarse unknowns)"), (144, "16-CTA cluster (243 coarse unknowns)")])
def test_single_sheet_matches_fp64_and_cuts_iterations(ctx_factory, nq, path):
    scene = scenes.precision_sheet(nq, seed=3)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = scene.sheets[0]["x"], scene.sheets[0]["v"]
    its = {}
    for coarse in (0, 1):
        ctx.set_state(x0, v0)
        st, _ = ctx.step(params(scene, coarse=coarse))
        assert st.converged == 1 and st.max_rel_residual <= 1e-10, path
        its[coarse] = st.max_iters
        if coarse:
            dv = ctx.get_dv().reshape(-1)
    (exact,) = fp64_dv(ctx, params(scene, coarse=1), ranges_of(scene))
    assert rel(dv, exact) < 1e-6, path
    print(f"{path}: CG iterations block-Jacobi {its[0]}, with the coarse correction {its[1]}")
    assert its[1] < 0.6 * its[0], (path, its)


def test_uneven_batch_matches_fp64_and_repeats_bit_for_bit(ctx_factory):
    """Sheets of 16-130 quads a side in one batched loop, each with its own coarse space."""
    scene = scenes.uneven_batch(12, seed=21, nq_range=(16, 130))
    ctx = ctx_factory(scene.sheets)
    x0 = np.concatenate([s["x"] for s in scene.sheets])
    v0 = np.concatenate([s["v"] for s in scene.sheets])
    p = params(scene, coarse=1)
    ctx.set_state(x0, v0)
    st, _ = ctx.step(p)
    assert st.converged == 12 and st.max_rel_residual <= 1e-10
    dv = ctx.get_dv().reshape(-1)
    it1, _, _ = ctx.instance_stats()
    ctx.set_state(x0, v0)
    ctx.step(p)
    assert np.array_equal(ctx.get_dv().reshape(-1), dv)
    p.use_graph = 0
    ctx.set_state(x0, v0)
    ctx.step(p)
    assert np.array_equal(ctx.get_dv().reshape(-1), dv)
    for (n0, n1), exact in zip(ranges_of(scene), fp64_dv(ctx, params(scene, coarse=1), ranges_of(scene))):
        assert rel(dv[3 * n0:3 * n1], exact) < 1e-6
    ctx.set_state(x0, v0)
    ctx.step(params(scene, coarse=0))
    it0, _, _ = ctx.instance_stats()
    assert it1.sum() < 0.8 * it0.sum(), (it0, it1)


def test_plain_fp32_and_tolerance_1e6_with_the_correction(ctx_factory):
    """The correction under plain FP32 PCG (its own recursive residual) and the mixed solver at
    the benchmark's 1e-6: both end, the mixed one at its FP64-checked tolerance."""
    scene = scenes.precision_sheet(64, seed=4)
    ctx = ctx_factory(scene.sheets)
    st, _ = ctx.step(params(scene, coarse=1, tol=1e-6))
    assert st.converged == 1 and st.max_rel_residual <= 1e-6
    st, _ = ctx.step(params(scene, coarse=1, tol=1e-6, precision=native.PREC_PLAIN_FP32), allow_unconverged=True)
    assert st.max_rel_residual < 1e-3
