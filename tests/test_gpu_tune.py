"""The autotuner (cs_tune): every launch shape of the batched SpMV computes the same bits, the
fastest is used by later steps, which then give the same dv bit for bit, and the preconditioner
the tuner reports is one it timed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native, scenes


def test_tuner_shapes_agree_and_the_choice_is_applied(ctx_factory):
    scene = scenes.windy_batch(24, 64, seed=501)
    scene.sheets += scenes.uneven_batch(6, seed=502, nq_range=(20, 130)).sheets  # some stay in the batched loop
    ctx = ctx_factory(scene.sheets)
    x0 = np.concatenate([s["x"] for s in scene.sheets])
    v0 = np.concatenate([s["v"] for s in scene.sheets])
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-8, max_iters=20000,
                           solver=native.SOLVER_BATCHED, advance=0)
    ctx.set_state(x0, v0)
    ctx.step(p)
    before = ctx.get_dv().copy()
    res = ctx.tune(p, reps=3)
    sums = {s["checksum"] for s in res["spmv"]}
    assert len(sums) == 1, "every SpMV launch shape must compute the same bits"
    assert all(s["ms"] > 0 for s in res["spmv"])
    best = res["spmv"][res["best_spmv"]]
    assert best["ms"] == min(s["ms"] for s in res["spmv"])
    info = ctx.solver_info()
    assert (info["spmv_threads_per_block"], info["spmv_slices_per_warp"], info["spmv_slots_loaded_together"]) == \
        (best["threads"], best["slices_per_warp"], best["unroll"])
    bp = res["precond"][res["best_precond"]]
    assert bp["ms"] == min(q["ms"] for q in res["precond"]) > 0
    assert (info["tuned_precond_degree"], info["tuned_coarse"]) == (bp["degree"], bp["coarse"])
    # both solve routes timed, the faster reported
    ms = res["solver_ms"]
    assert ms["auto"] > 0 and ms["batched"] > 0
    assert res["best_solver"] == ("auto" if ms["auto"] <= ms["batched"] else "batched")
    # the same step with the tuned shape: the same dv bits (graph rebuilt after tuning)
    ctx.set_state(x0, v0)
    ctx.step(p)
    assert np.array_equal(ctx.get_dv(), before)
    p.use_graph = 0
    ctx.set_state(x0, v0)
    ctx.step(p)
    assert np.array_equal(ctx.get_dv(), before)
