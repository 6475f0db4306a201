"""GPU tests of the learned warm start's tensor-core path."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native


def to_bf16_bits(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def from_bf16_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("K,N", [(16, 16), (32, 64), (64, 64), (128, 64), (64, 128), (128, 128)])
def test_tcgen05_tile_gemm_matches_fp64(K, N):
    lib = native.load_library()
    rng = np.random.default_rng(K * 1000 + N)
    A = to_bf16_bits(rng.normal(size=(128, K)))
    B = to_bf16_bits(rng.normal(size=(N, K)))
    D = np.zeros((128, N), np.float32)
    st = lib.cs_tc_gemm_check(A.ctypes.data, B.ctypes.data, D.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), K, N)
    assert st == native.CS_OK
    ref = from_bf16_bits(A).astype(np.float64) @ from_bf16_bits(B).astype(np.float64).T
    assert np.abs(D - ref).max() / np.abs(ref).max() < 1e-5


# --- the network: gradients against the FP64 oracle, training, and the warm start's gain ----
import mlp_oracle  # noqa: E402
from clothsimulator_b200 import scenes  # noqa: E402


def recorded_ctx(scene, steps, slots=None, tol=1e-8, seed=3):
    ctx = native.Context(0)
    ctx.load(scene.sheets)
    ctx.mlp_init(slots or steps, seed)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=tol, max_iters=8000)
    for t in range(steps):
        ctx.assemble(p)
        ctx.mlp_record(t, 0)
        ctx.step(p)
        ctx.mlp_record(t, 1)
        p.warm_start = native.WARM_PREVIOUS
    ctx.mlp_fit_normalization(steps)
    return ctx, p


def batch_neighbours(scene):
    nb, off = [], 0
    for s in scene.sheets:
        n = s["x"].shape[0]
        nb += [j + off for j in mlp_oracle.neighbours(s["fx"], n)]
        off += n
    return nb


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_mlp_gradient_and_prediction_match_fp64_oracle():
    scene = scenes.windy_batch(3, 8, seed=5)
    ctx, p = recorded_ctx(scene, 2)
    w = ctx.mlp_get_weights()
    feat, target = ctx.mlp_get_record(1)
    nb = batch_neighbours(scene)
    g, loss = ctx.mlp_gradient(1, 0, 3)
    loss_ref, g_ref, _ = mlp_oracle.loss_and_grad(w, feat.astype(np.float64), target.astype(np.float64), nb)
    assert abs(loss - loss_ref) / loss_ref < 1e-4
    assert rel(g, g_ref) < 2e-3
    # prediction for the current system
    ctx.assemble(p)
    pred = ctx.mlp_predict()
    feat_now = None
    ctx.mlp_record(0, 0)
    feat_now, _ = ctx.mlp_get_record(0)
    ref = mlp_oracle.predict(w, feat_now.astype(np.float64), nb)
    assert rel(pred, ref) < 1e-4
    ctx.close()


def test_energy_gradient_matches_fp64_oracle():
    """The energy-norm loss (sin^2 of the A-angle between prediction and solution) and its
    gradient (cs_mlp_energy_gradient) against the FP64 restatement on the batch's system at the
    current state: loss within 1e-4, gradient within 2e-3, over the whole batch and over one
    sheet of it."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    scene = scenes.windy_batch(3, 8, seed=5)
    ctx, p = recorded_ctx(scene, 2)
    p.tol = 1e-11
    w = ctx.mlp_get_weights()
    nb = batch_neighbours(scene)
    ranges, off = [], 0
    for s in scene.sheets:
        ranges.append((off, off + s["x"].shape[0]))
        off += s["x"].shape[0]
    for s0, s1 in ((0, 3), (1, 2)):
        g, loss = ctx.mlp_energy_gradient(p, s0, s1)
        # the same state's features and system (the call changed neither the state nor B.warm)
        ctx.assemble(p)
        ctx.mlp_record(0, 0)
        feat, _ = ctx.mlp_get_record(0)
        rp, ci, val, b = ctx.system()
        n = rp.shape[0] - 1
        A = sp.bsr_matrix((val.astype(np.float64), ci, rp), shape=(3 * n, 3 * n)).tocsr()
        b64 = b.astype(np.float64)
        dvs = spl.spsolve(A.tocsc(), b64)
        n0, n1 = ranges[s0][0], ranges[s1 - 1][1]
        Asub = A[3 * n0:3 * n1, 3 * n0:3 * n1]
        sub_ranges = [(a - n0, z - n0) for a, z in ranges[s0:s1]]
        sub_nb = [j - n0 for j in nb[n0:n1]]
        loss_ref, g_ref, _ = mlp_oracle.energy_loss_and_grad(w, feat[n0:n1].astype(np.float64), Asub,
                                                             b64[3 * n0:3 * n1], dvs[3 * n0:3 * n1], sub_ranges, sub_nb)
        assert abs(loss - loss_ref) / abs(loss_ref) < 1e-4, (s0, s1, loss, loss_ref)
        assert rel(g, g_ref) < 2e-3, (s0, s1)
    ctx.close()


def test_energy_training_step_lowers_the_energy_loss():
    """cs_mlp_train_step along a trajectory lowers the energy-norm loss (in [0, 1]) at the
    trajectory's first state, and the step it takes equals cs_step's (same solve, same update:
    x, v bit for bit)."""
    scene = scenes.windy_batch(8, 12, seed=6)
    ctx, p = recorded_ctx(scene, 4)
    x, v = ctx.get_state()
    prev = ctx.get_dv()
    _, before = ctx.mlp_energy_gradient(p, 0, 8)
    twin = native.Context(0)
    twin.load(scene.sheets)
    twin.set_state(x, v)
    twin.set_warm_start(prev)
    q = native.StepParams.from_buffer_copy(p)
    q.use_graph = 0
    for t in range(24):
        st, loss = ctx.mlp_train_step(p, lr=2e-3, sheets_per_batch=2, seed=t)
        twin.step(q)
        assert st.converged == 8 and 0.0 <= loss <= 1.0
    xa, va = ctx.get_state()
    xb, vb = twin.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    # the loss at the trajectory's first state, before and after the training
    ctx.set_state(x, v)
    ctx.set_warm_start(prev)
    _, after = ctx.mlp_energy_gradient(p, 0, 8)
    print(f"energy loss at the first state: {before:.4f} -> {after:.4f}")
    assert after < 0.8 * before
    twin.close()
    ctx.close()


def test_mlp_training_reduces_loss():
    scene = scenes.windy_batch(8, 12, seed=6)
    ctx, _ = recorded_ctx(scene, 4)
    losses = ctx.mlp_train(4, 40, lr=2e-3, sheets_per_batch=2, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0]
    ctx.close()


def test_learned_warm_start_converges_and_reports_gain():
    """Train on one set of seeded trajectories, evaluate on held-out ones: every sheet must
    reach the FP64-checked tolerance, and the learned start's iterations are reported next to
    the zero and previous-dv starts (the gain the network buys)."""
    train = scenes.windy_batch(16, 16, seed=11)
    ctx, _ = recorded_ctx(train, 12, tol=1e-7)
    ctx.mlp_train(12, 30, lr=2e-3, sheets_per_batch=4, seed=2)
    w = ctx.mlp_get_weights()
    ctx.close()
    held = scenes.windy_batch(16, 16, seed=99)
    iters = {}
    for mode in (native.WARM_ZERO, native.WARM_PREVIOUS, native.WARM_LEARNED):
        ev = native.Context(0)
        ev.load(held.sheets)
        ev.mlp_init(0, 0)
        ev.mlp_set_weights(w)
        p = native.step_params(held.dt, held.gravity, held.handle_stiffness, tol=1e-6, max_iters=8000)
        total = 0
        for t in range(8):
            st, _ = ev.step(p)
            assert st.converged == 16
            if t >= 3:
                total += st.total_iters
            p.warm_start = mode
        iters[mode] = total
        ev.close()
    print("total CG iterations over 5 held-out steps: zero %d, previous %d, learned %d" % (
        iters[native.WARM_ZERO], iters[native.WARM_PREVIOUS], iters[native.WARM_LEARNED]))
    # the guard discards starts worse than zero, so the learned start costs at most noise-level
    # extra iterations (its gain on this workload is nil: the iterations are set by conditioning)
    assert iters[native.WARM_LEARNED] <= 1.01 * iters[native.WARM_ZERO]
