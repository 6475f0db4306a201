"""Cluster-resident PCG (one thread-block cluster per sheet, the system in distributed shared
memory) against the CPU oracle and against the batched loop on the same state.

Tolerances (norm-wise relative):
  * dv of a solve to an FP64-checked relative residual of 1e-10 against an FP64 direct solve
    of the same FP32 system: 1e-6 (as for the batched loop);
  * plain FP32 PCG: the FP64-checked residual of the resident and batched solvers within a
    factor 10 of each other (FP32 rounding differs with the summation order);
  * iteration counts of the resident and batched solvers on identical systems: within 10 %
    (same iteration, different summation order of the dot products).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import pyoracle
from clothsimulator_b200 import native, scenes


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def params_for(scene, **kw):
    kw.setdefault("tol", 1e-10)
    kw.setdefault("max_iters", 20000)
    kw.setdefault("advance", 0)
    return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, **kw)


def oracle_dv(scene, sheet):
    c = pyoracle.Cloth(sheet, pyoracle.Material(sheet["material"], "float"))
    c.assemble(scenes.step_params(scene, sheet))
    dv, _ = c.solve(pyoracle.METHOD_LLT64)
    return dv


def split_dv(ctx, scene):
    dv = ctx.get_dv().reshape(-1, 3)
    out, o = [], 0
    for s in scene.sheets:
        n = s["x"].shape[0]
        out.append(dv[o:o + n].reshape(-1))
        o += n
    return out


def initial_state(scene):
    return (np.concatenate([s["x"] for s in scene.sheets]), np.concatenate([s["v"] for s in scene.sheets]))


def test_plan_covers_sheets_that_fit(ctx_factory):
    scene = scenes.windy_batch(6, 64, seed=11)
    ctx = ctx_factory(scene.sheets)
    info = ctx.solver_info()
    assert info["resident_sheets"] == 6
    # 8, 9 or 10 CTAs per cluster: whichever keeps more SMs busy for this plan
    assert info["ctas_per_cluster"] in (8, 9, 10) and info["clusters"] >= 1
    assert info["threads_per_cta"] % 32 == 0 and info["threads_per_cta"] <= 768
    # a 128x128 sheet needs more than 24 slices per CTA: it stays in the batched loop
    big = scenes.windy_batch(1, 128, seed=12).sheets + scenes.windy_batch(2, 32, seed=13).sheets
    ctx2 = ctx_factory(big)
    assert ctx2.solver_info()["resident_sheets"] == 2


def test_resident_solve_matches_oracle(ctx_factory):
    scene = scenes.windy_batch(3, 32, seed=21)
    scene.sheets += scenes.windy_batch(1, 64, seed=22).sheets
    ctx = ctx_factory(scene.sheets)
    assert ctx.solver_info()["resident_sheets"] == 4
    stats, _ = ctx.step(params_for(scene))
    assert stats.converged == 4
    for s, dv in zip(scene.sheets, split_dv(ctx, scene)):
        assert rel(dv, oracle_dv(scene, s)) < 1e-6


def test_resident_and_batched_agree(ctx_factory):
    scene = scenes.windy_batch(4, 32, seed=31)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    res = {}
    for solver in (native.SOLVER_AUTO, native.SOLVER_BATCHED):
        ctx.set_state(x0, v0)
        # the same preconditioner on both routes: block-Jacobi, no coarse correction
        stats, _ = ctx.step(params_for(scene, solver=solver, coarse=0))
        it, rr, fl = ctx.instance_stats()
        res[solver] = (ctx.get_dv().copy(), it.copy(), rr.copy(), fl.copy(), stats.loop_trips)
    dva, ita, rra, fla, tripa = res[native.SOLVER_AUTO]
    dvb, itb, rrb, flb, tripb = res[native.SOLVER_BATCHED]
    assert np.all(fla & 1) and np.all(flb & 1)
    assert np.all(rra <= 1e-10) and np.all(rrb <= 1e-10)
    assert rel(dva, dvb) < 1e-6
    assert np.all(np.abs(ita - itb) <= 0.1 * itb + 2)
    # every sheet resident: the batched loop only runs its closing trip
    assert tripa <= 1 < tripb


def test_resident_plain_fp32_matches_batched_plain(ctx_factory):
    scene = scenes.windy_batch(4, 32, seed=41)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    res = {}
    for solver in (native.SOLVER_AUTO, native.SOLVER_BATCHED):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, tol=1e-6, precision=native.PREC_PLAIN_FP32, solver=solver, coarse=0),
                 allow_unconverged=True)
        res[solver] = ctx.instance_stats()
    ita, rra, fla = res[native.SOLVER_AUTO]
    itb, rrb, flb = res[native.SOLVER_BATCHED]
    assert np.all(ita > 0) and np.all(np.abs(ita - itb) <= 0.1 * itb + 2)
    # the FP64 check of the plain solver's answer: converged exactly when it met tol
    assert np.array_equal((fla & 1) > 0, rra <= 1e-6)
    assert np.all(rra < 1e-3) and np.all(np.abs(np.log10(rra / rrb)) < 1.0)


def test_resident_warm_start_and_guard(ctx_factory):
    scene = scenes.windy_batch(4, 32, seed=51)
    ctx = ctx_factory(scene.sheets)
    p = params_for(scene, tol=1e-8, advance=1)
    ctx.step(p)
    p.warm_start = native.WARM_PREVIOUS
    stats, _ = ctx.step(p)
    assert stats.converged == 4
    # a warm start far worse than zero must be discarded, and the solve still converges
    ctx.set_warm_start(np.full((ctx.n, 3), 1e3, np.float32))
    p.warm_start = native.WARM_GIVEN
    stats, _ = ctx.step(p)
    assert stats.converged == 4 and stats.warm_rejected == 4


def test_resident_iteration_cap_returns(ctx_factory):
    scene = scenes.windy_batch(3, 32, seed=61)
    ctx = ctx_factory(scene.sheets)
    stats, st = ctx.step(params_for(scene, max_iters=5), allow_unconverged=True)
    it, rr, fl = ctx.instance_stats()
    assert st == native.CS_ERR_NOT_CONVERGED
    assert np.all(it <= 5) and np.all(fl & 8) and not np.any(fl & 1)


def test_resident_is_deterministic(ctx_factory):
    scene = scenes.windy_batch(3, 32, seed=71)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    out = []
    for _ in range(2):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, tol=1e-6))
        out.append(ctx.get_dv().copy())
    assert np.array_equal(out[0], out[1])


def test_mixed_resident_and_batched_batch(ctx_factory):
    sheets = scenes.windy_batch(1, 128, seed=81).sheets + scenes.windy_batch(2, 32, seed=82).sheets
    scene = scenes.Scene("mixed", sheets, dt=1.0 / 100, steps=1)
    ctx = ctx_factory(scene.sheets)
    assert ctx.solver_info()["resident_sheets"] == 2
    stats, _ = ctx.step(params_for(scene))
    assert stats.converged == 3
    for s, dv in zip(scene.sheets, split_dv(ctx, scene)):
        assert rel(dv, oracle_dv(scene, s)) < 1e-6


# Strip-local Chebyshev preconditioner (precond_degree 3..15, odd): a different but fixed SPD
# preconditioner, so the solution must still meet the FP64-checked tolerance and match the
# direct solve; the iteration counts must fall well below block-Jacobi's.

@pytest.mark.parametrize("degree", [3, 5, 7])
def test_chebyshev_resident_matches_oracle(ctx_factory, degree):
    scene = scenes.windy_batch(3, 32, seed=21)
    scene.sheets += scenes.windy_batch(1, 64, seed=22).sheets
    ctx = ctx_factory(scene.sheets)
    assert ctx.solver_info()["resident_sheets"] == 4
    x0, v0 = initial_state(scene)
    it = {}
    for deg in (1, degree):
        ctx.set_state(x0, v0)
        stats, _ = ctx.step(params_for(scene, precond_degree=deg))
        assert stats.converged == 4
        it[deg], rr, fl = ctx.instance_stats()
        assert np.all(rr <= 1e-10)
        for s, dv in zip(scene.sheets, split_dv(ctx, scene)):
            assert rel(dv, oracle_dv(scene, s)) < 1e-6
    # degree 3 needs about half of block-Jacobi's iterations, 5 and 7 about a third
    bound = 0.7 if degree == 3 else 0.55
    assert it[degree].sum() <= bound * it[1].sum(), (it[degree], it[1])


def test_chebyshev_plain_fp32_and_determinism(ctx_factory):
    scene = scenes.windy_batch(3, 32, seed=71)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    out = []
    for _ in range(2):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, tol=1e-6, precond_degree=5))
        out.append(ctx.get_dv().copy())
    assert np.array_equal(out[0], out[1])
    ctx.set_state(x0, v0)
    ctx.step(params_for(scene, tol=1e-6, precision=native.PREC_PLAIN_FP32, precond_degree=5), allow_unconverged=True)
    it, rr, fl = ctx.instance_stats()
    assert np.all(it > 0) and np.all(rr < 1e-3)
    assert np.array_equal((fl & 1) > 0, rr <= 1e-6)


def test_chebyshev_degree_is_ignored_by_batched_loop(ctx_factory):
    scene = scenes.windy_batch(2, 32, seed=91)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    res = []
    for deg in (1, 5):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, solver=native.SOLVER_BATCHED, precond_degree=deg))
        res.append((ctx.get_dv().copy(), ctx.instance_stats()[0].copy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_chebyshev_degree_validation(ctx_factory):
    scene = scenes.windy_batch(1, 16, seed=92)
    ctx = ctx_factory(scene.sheets)
    for bad in (-1, 2, 4, 17):
        st = ctx.lib.cs_step(ctx.h, native.ctypes.byref(params_for(scene, precond_degree=bad)), None)
        assert st == native.CS_ERR_INVALID_ARG, bad


def test_resident_blocks_accounting(ctx_factory):
    """cs_get_resident_blocks: the resident sheets' pattern blocks (the system's, with no
    proximities), the strip-local ones among them, and the power iterations per solve."""
    scene = scenes.windy_batch(3, 32, seed=93)
    scene.sheets += scenes.windy_batch(1, 64, seed=94).sheets
    ctx = ctx_factory(scene.sheets)
    rb = ctx.resident_blocks()
    assert ctx.solver_info()["resident_sheets"] == 4
    assert rb["blocks"] == ctx.sizes[6]
    # most blocks couple rows of the same strip; the strips' borders couple the rest
    assert 0.5 * rb["blocks"] < rb["local_blocks"] < rb["blocks"]
    assert rb["power_iters"] == 10


def test_chebyshev_falls_back_on_thin_strips(ctx_factory):
    """Sheets split into strips that keep less than 0.62 of their blocks (16x16 sheets over a
    cluster) solve with block-Jacobi even when the Chebyshev preconditioner is asked for: the
    same iterations and the same dv bits as precond_degree 1."""
    scene = scenes.windy_batch(3, 16, seed=95)
    ctx = ctx_factory(scene.sheets)
    rb = ctx.resident_blocks()
    assert rb["local_blocks"] < 0.62 * rb["blocks"]
    x0, v0 = initial_state(scene)
    res = []
    for deg in (1, 3):
        ctx.set_state(x0, v0)
        stats, _ = ctx.step(params_for(scene, precond_degree=deg))
        assert stats.converged == 3
        res.append((ctx.get_dv().copy(), ctx.instance_stats()[0].copy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


# Coarse-space correction (coarse=1 with the Chebyshev preconditioner): each CTA's strip cut
# into geometric segments, one coarse unknown per (segment, component), the coarse matrix
# R A R^T inverted per sheet and step; an additive SPD term, so the solve must still meet the
# FP64-checked tolerance and match the direct solve, in fewer iterations.

def test_coarse_correction_matches_oracle_and_cuts_iterations(ctx_factory):
    scene = scenes.windy_batch(5, 64, seed=301)
    scene.sheets += scenes.windy_batch(2, 48, seed=302).sheets
    ctx = ctx_factory(scene.sheets)
    assert ctx.solver_info()["resident_sheets"] == len(scene.sheets)
    x0, v0 = initial_state(scene)
    it = {}
    for coarse in (0, 1):
        ctx.set_state(x0, v0)
        stats, _ = ctx.step(params_for(scene, precond_degree=3, coarse=coarse))
        assert stats.converged == len(scene.sheets)
        it[coarse], rr, fl = ctx.instance_stats()
        assert np.all(rr <= 1e-10)
        for s, dv in zip(scene.sheets, split_dv(ctx, scene)):
            assert rel(dv, oracle_dv(scene, s)) < 1e-6
    print("CG iterations without / with the coarse correction:", it[0].tolist(), it[1].tolist())
    assert it[1].sum() <= 0.8 * it[0].sum(), (it[1], it[0])


def test_coarse_correction_deterministic_and_guarded(ctx_factory):
    scene = scenes.windy_batch(4, 64, seed=311)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    out = []
    for _ in range(2):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, tol=1e-6, precond_degree=3, coarse=1))
        out.append((ctx.get_dv().copy(), ctx.instance_stats()[0].copy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    # a warm start worse than the zero guess is discarded: the solve restarts from dv = 0
    ctx.set_state(x0, v0)
    ctx.set_warm_start(np.full((ctx.n, 3), 1e3, np.float32))
    stats, _ = ctx.step(params_for(scene, precond_degree=3, coarse=1, warm_start=native.WARM_GIVEN))
    it, rr, fl = ctx.instance_stats()
    assert stats.converged == 4 and stats.warm_rejected == 4 and np.all(fl & 2) and np.all(rr <= 1e-10)
    for s, dv in zip(scene.sheets, split_dv(ctx, scene)):
        assert rel(dv, oracle_dv(scene, s)) < 1e-6
    # the exact solution as the warm start needs no iteration
    ctx.set_warm_start(ctx.get_dv())
    ctx.set_state(x0, v0)
    stats, _ = ctx.step(params_for(scene, tol=1e-6, precond_degree=3, coarse=1, warm_start=native.WARM_GIVEN))
    assert stats.converged == 4 and stats.max_iters == 0 and stats.warm_rejected == 0


def test_coarse_correction_plain_fp32(ctx_factory):
    scene = scenes.windy_batch(3, 64, seed=321)
    ctx = ctx_factory(scene.sheets)
    stats, _ = ctx.step(params_for(scene, tol=1e-6, precision=native.PREC_PLAIN_FP32, precond_degree=3, coarse=1),
                        allow_unconverged=True)
    it, rr, fl = ctx.instance_stats()
    assert np.all(it > 0) and np.all(rr < 1e-3)
    assert np.array_equal((fl & 1) > 0, rr <= 1e-6)


def test_coarse_flag_inert_without_chebyshev(ctx_factory):
    """With block-Jacobi (degree 1) the coarse flag changes nothing, bit for bit."""
    scene = scenes.windy_batch(2, 64, seed=331)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    res = []
    for coarse in (0, 1):
        ctx.set_state(x0, v0)
        ctx.step(params_for(scene, precond_degree=1, coarse=coarse))
        res.append((ctx.get_dv().copy(), ctx.instance_stats()[0].copy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


@pytest.mark.parametrize("route", ["resident_coarse", "resident_jacobi", "batched"])
def test_galerkin_scaled_warm_start(ctx_factory, route):
    """warm_scale: warm starts of 4 and -2 times the solution (exact in FP32) have residuals of
    3 ||b||, which the guard discards; their Galerkin multiples (d.b / d.A d = 1/4, -1/2) are the
    solution, which the guard keeps, and the solve then needs far fewer iterations than from
    zero."""
    scene = scenes.windy_batch(4, 24, seed=71)
    ctx = ctx_factory(scene.sheets)
    x0 = np.concatenate([s["x"] for s in scene.sheets])
    v0 = np.concatenate([s["v"] for s in scene.sheets])
    kw = {"resident_coarse": dict(precond_degree=3, coarse=1), "resident_jacobi": dict(precond_degree=1, coarse=0),
          "batched": dict(solver=native.SOLVER_BATCHED)}[route]
    ctx.set_state(x0, v0)
    ctx.step(params_for(scene, tol=1e-11, **kw))
    exact = ctx.get_dv().copy()
    ctx.set_state(x0, v0)
    ctx.step(params_for(scene, tol=1e-7, **kw))
    it_zero, _, _ = ctx.instance_stats()
    for scale in (0, 1):
        for mult in (4.0, -2.0):
            ctx.set_state(x0, v0)
            ctx.set_warm_start(mult * exact)
            st, _ = ctx.step(params_for(scene, tol=1e-7, warm_start=native.WARM_PREVIOUS, warm_scale=scale, **kw))
            it, rr, fl = ctx.instance_stats()
            assert st.converged == 4 and np.all(rr <= 1e-7)
            assert rel(ctx.get_dv(), exact) < 1e-5
            if scale == 0:
                assert np.all(fl & 2), "a start of 4x or -2x the solution is worse than zero"
            else:
                assert not np.any(fl & 2)
                assert np.all(it <= 0.5 * it_zero), (it, it_zero)


def test_converged_warm_start_reports_an_fp64_residual(ctx_factory):
    """A warm start of twice the solution, Galerkin-scaled (factor 1/2), meets a loose tolerance
    with no CG iteration.  The resident solver forms the scaled start's residual as (1 - a) b + a r
    from the scale pass's residual r without an SpMV; a solve that would end on that residual
    takes an FP64 residual of the scaled start first.  So the residual it reports is an FP64 one:
    it agrees with the batched loop's, which always computes the scaled start's FP64 residual,
    to 1e-4 relative (an affine residual built from the FP32 copy of r would miss by percents:
    the scaled residual is the size of the solution's FP32 rounding)."""
    scene = scenes.windy_batch(4, 24, seed=73)
    ctx = ctx_factory(scene.sheets)
    x0, v0 = initial_state(scene)
    ctx.set_state(x0, v0)
    ctx.step(params_for(scene, tol=1e-12, precond_degree=3, coarse=1))
    exact = ctx.get_dv().copy()
    rr = {}
    for route, kw in (("resident_coarse", dict(precond_degree=3, coarse=1)),
                      ("resident_jacobi", dict(precond_degree=1, coarse=0)),
                      ("batched", dict(solver=native.SOLVER_BATCHED))):
        ctx.set_state(x0, v0)
        ctx.set_warm_start(2.0 * exact)
        st, _ = ctx.step(params_for(scene, tol=1e-3, warm_start=native.WARM_PREVIOUS, warm_scale=1, **kw))
        it, res, fl = ctx.instance_stats()
        assert st.converged == 4 and np.all(it == 0) and not np.any(fl & 2), (route, it, fl)
        assert rel(ctx.get_dv(), exact) < 1e-5, route
        rr[route] = res.copy()
    for route in ("resident_coarse", "resident_jacobi"):
        assert np.all(np.abs(rr[route] - rr["batched"]) <= 1e-4 * rr["batched"]), (route, rr[route], rr["batched"])
