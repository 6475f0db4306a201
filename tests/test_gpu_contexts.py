"""Several contexts in one process, loaded with batches of different sizes.

The limit on a kernel's dynamic shared memory belongs to the kernel function, not to a
context.  The assembly gather (slot accumulators per row width), the cluster-resident solver
(a strip of the sheet's panels per CTA) and its coarse set-up size their shared memory by the
batch, so a context loaded after another must not lower what the earlier one launches with:
each context still steps, captured in its CUDA graph, after a smaller batch was loaded."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native, scenes


def params_for(scene, **kw):
    kw.setdefault("tol", 1e-6)
    kw.setdefault("max_iters", 20000)
    kw.setdefault("advance", 0)
    return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, **kw)


def test_larger_batches_step_after_a_smaller_one_is_loaded(ctx_factory):
    # widest rows (17 block slots) and a sheet too large for a cluster: the batched loop
    irregular = scenes.large_irregular(120, seed=5)
    # 64x64 sheets: the resident kernel with a near-full strip of panels per CTA
    windy = scenes.windy_batch(2, 64, seed=6)
    # loaded last: 13 slots per row, small resident strips
    small = scenes.windy_batch(2, 16, seed=7)
    big = [(irregular, ctx_factory(irregular.sheets)), (windy, ctx_factory(windy.sheets))]
    ctx_small = ctx_factory(small.sheets)
    st, _ = ctx_small.step(params_for(small, precond_degree=3, coarse=1))
    assert st.converged == 2
    for scene, ctx in big:
        for graph in (1, 0):
            p = params_for(scene, precond_degree=3, coarse=1)
            p.use_graph = graph
            st, _ = ctx.step(p)
            it, rr, fl = ctx.instance_stats()
            assert st.converged == len(scene.sheets) and np.all(rr <= 1e-6), (graph, rr)
