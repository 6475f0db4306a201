"""Data-parallel training of the learned warm start (clothsimulator_b200.training) on the GPU.

* one rank with an identity all-reduce reproduces cs_mlp_train's weights bit for bit (same
  minibatch order, gradient kernels and Adam update);
* two ranks in lockstep (two contexts on one GPU, a host-side all-reduce of their device
  gradients) holding the same trajectories end with the single rank's weights bit for bit
  ((g + g) / 2 = g), and two ranks on different trajectories end with identical weights.
"""
import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native, scenes, training

SLOTS, SHEETS, NQ = 3, 6, 12


def recorded_ctx(seed):
    sc = scenes.windy_batch(SHEETS, NQ, seed=seed)
    ctx = native.Context(0).load(sc.sheets)
    ctx.mlp_init(SLOTS, 1)
    p = native.step_params(sc.dt, sc.gravity, sc.handle_stiffness, tol=1e-7, max_iters=8000)
    ctx.step(p, allow_unconverged=True)
    p.warm_start = native.WARM_PREVIOUS
    for t in range(SLOTS):
        ctx.assemble(p)
        ctx.mlp_record(t, 0)
        ctx.step(p, allow_unconverged=True)
        ctx.mlp_record(t, 1)
    return ctx


def test_single_rank_matches_mlp_train():
    a, b = recorded_ctx(11), recorded_ctx(11)
    a.mlp_fit_normalization(SLOTS)
    la = a.mlp_train(SLOTS, 3, lr=1e-3, sheets_per_batch=2, seed=5)
    lb = training.train_data_parallel(b, SLOTS, SHEETS, 3, 1e-3, 2, 5, allreduce_sum=None, world=1)
    assert np.array_equal(a.mlp_get_weights(), b.mlp_get_weights())
    assert np.allclose(la, lb, rtol=1e-5)
    a.close()
    b.close()


class LockstepGroup:
    """A two-rank all-reduce between threads: sums the ranks' tensors in place."""

    def __init__(self):
        self.bar = threading.Barrier(2)
        self.slot = [None, None]

    def allreduce(self, rank):
        def fn(t):
            torch.cuda.synchronize()
            self.slot[rank] = t
            self.bar.wait()
            if rank == 0:
                s = self.slot[0] + self.slot[1]
                self.slot[0].copy_(s)
                self.slot[1].copy_(s)
                torch.cuda.synchronize()
            self.bar.wait()
        return fn

    def sum_host(self, rank):
        def fn(a):
            self.slot[rank] = a
            self.bar.wait()
            out = self.slot[0] + self.slot[1]
            self.bar.wait()
            return out
        return fn


def run_two(seeds):
    ctxs = [recorded_ctx(s) for s in seeds]
    g = LockstepGroup()
    errs = []

    def work(r):
        try:
            training.train_data_parallel(ctxs[r], SLOTS, SHEETS, 2, 1e-3, 2, 5, allreduce_sum=g.allreduce(r),
                                         world=2, sum_host=g.sum_host(r))
        except Exception as e:  # surfaced below
            errs.append(e)
            g.bar.abort()

    th = [threading.Thread(target=work, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(300)
    assert not errs, errs
    w = [c.mlp_get_weights() for c in ctxs]
    for c in ctxs:
        c.close()
    return w


def test_two_ranks_same_data_equal_one_rank():
    w2 = run_two([21, 21])
    one = recorded_ctx(21)
    training.train_data_parallel(one, SLOTS, SHEETS, 2, 1e-3, 2, 5, allreduce_sum=None, world=1)
    w1 = one.mlp_get_weights()
    one.close()
    assert np.array_equal(w2[0], w2[1]) and np.array_equal(w2[0], w1)


def test_two_ranks_different_data_agree():
    w = run_two([31, 32])
    assert np.array_equal(w[0], w[1])


def test_energy_single_rank_matches_train_step():
    """The data-parallel energy step (cs_mlp_energy_begin / _gradient_device / apply / _end) with
    one rank reproduces cs_mlp_train_step bit for bit: weights, state and losses."""
    a, b = recorded_ctx(13), recorded_ctx(13)
    for c in (a, b):
        c.mlp_fit_normalization(SLOTS)
    sc = scenes.windy_batch(SHEETS, NQ, seed=13)
    p = native.step_params(sc.dt, sc.gravity, sc.handle_stiffness, tol=1e-7, max_iters=8000,
                           warm_start=native.WARM_PREVIOUS)
    for t in range(4):
        _, la = a.mlp_train_step(p, lr=1e-3, sheets_per_batch=2, seed=40 + t)
        _, lb = training.energy_step_data_parallel(b, p, SHEETS, 1e-3, 2, 40 + t, allreduce_sum=None, world=1,
                                                   allow_unconverged=False)
        assert abs(la - lb) <= 1e-6 * max(1.0, abs(la))
    assert np.array_equal(a.mlp_get_weights(), b.mlp_get_weights())
    xa, va = a.get_state()
    xb, vb = b.get_state()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
    a.close()
    b.close()
