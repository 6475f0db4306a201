"""The multi-rank path of bench.py on CPU: two gloo ranks, one process each, as torchrun
launches them on two GPUs.  Sheets are independent, so the ranks exchange no data; what is
checked is the plumbing around the solve: the barrier, the max over ranks of the device
times that the whole-job value is computed from, per-rank workloads of equal size drawn
from distinct seeds (weak scaling), and training seeds disjoint from every evaluated seed.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    from clothsimulator_b200 import scenes

    group = bench.RankGroup(timeout_s=60)
    assert (group.rank, group.world) == (rank, world)
    scene = scenes.windy_batch(4, 8, seed=bench.eval_seed(rank))
    # a rank-dependent "device time": the job's time is the slowest rank's
    ms = 100.0 + 25.0 * rank
    group.barrier()
    ms_max = group.max(ms)
    group.barrier()
    out[rank] = {
        "ms_max": ms_max,
        "nodes": scene.n_nodes,
        "first_x": scene.sheets[0]["x"][:, 2].copy(),
        "stiffness": scene.sheets[0]["material"]["stretching_mult"],
        "value": bench.aggregate_value(scene.n_nodes, 10, world, ms_max),
    }
    group.close()


@pytest.mark.timeout(180)
def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        res = dict(out)
    # every rank sees the slowest rank's time
    assert res[0]["ms_max"] == res[1]["ms_max"] == 125.0
    # weak scaling: equal work per rank, different sheets
    assert res[0]["nodes"] == res[1]["nodes"]
    assert not np.array_equal(res[0]["first_x"], res[1]["first_x"])
    assert res[0]["stiffness"] != res[1]["stiffness"]
    # whole-job value: all ranks' node-steps over the slowest rank's time
    assert res[0]["value"] == pytest.approx(2 * res[0]["nodes"] * 10 / 0.125)


def test_seed_sets_are_disjoint():
    sys.path.insert(0, ROOT)
    import bench

    evals = {bench.eval_seed(r) for r in range(32)}
    trains = {bench.train_seed(r) for r in range(32)}
    assert len(evals) == len(trains) == 32 and not (evals & trains)


def test_single_rank_group_is_local():
    sys.path.insert(0, ROOT)
    import bench

    saved = {k: os.environ.pop(k, None) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    try:
        g = bench.RankGroup()
        assert (g.rank, g.world, g.dist) == (0, 1, None)
        assert g.max(3.5) == 3.5
        g.barrier()
        g.close()
    finally:
        for k, v in saved.items():
            if v is not None:
                os.environ[k] = v


class FakeTrainingContext:
    """Stands in for native.Context in train_data_parallel on CPU: parameters w, gradient of
    0.5 |w - target|^2 with a target per (rank, slot, minibatch), plain descent as the step."""

    def __init__(self, rank, n):
        import torch

        self.rank, self.w = rank, np.zeros(n, np.float32)
        self.torch_device = torch.device("cpu")
        self.moments = None

    def target(self, rank, slot, s0):
        return np.full(self.w.shape, 0.1 * (1 + rank) + 0.01 * slot + 0.001 * s0, np.float32)

    def mlp_moments(self, n_slots):
        return np.arange(38, dtype=np.float64) * (1 + self.rank), 10 * (1 + self.rank)

    def mlp_set_moments(self, sums, count):
        self.moments = (np.array(sums), count)

    def mlp_gradient_device(self, slot, s0, s1, grad):
        g = self.w - self.target(self.rank, slot, s0)
        grad.numpy()[:] = g
        return float(0.5 * (g * g).sum())

    def mlp_apply_gradient(self, grad, lr):
        self.w = (self.w - np.float32(lr) * grad.numpy()).astype(np.float32)


def _dp_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from clothsimulator_b200 import native, training

    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    ctx = FakeTrainingContext(rank, native.MLP_TRAINED)

    def sum_host(a):
        t = torch.from_numpy(np.array(a, np.float64))
        dist.all_reduce(t)
        return t.numpy()

    training.train_data_parallel(ctx, 2, 5, 2, 0.5, 2, 9, allreduce_sum=dist.all_reduce, world=world,
                                 sum_host=sum_host)
    out[rank] = {"w": ctx.w.copy(), "moments": ctx.moments}
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_data_parallel_training_two_gloo_ranks():
    """train_data_parallel over two gloo ranks: identical parameters on both, equal to serial
    descent on the averaged gradients, and the normalisation from the summed moments."""
    sys.path.insert(0, ROOT)
    from clothsimulator_b200 import native, training

    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_dp_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        res = dict(out)
    assert np.array_equal(res[0]["w"], res[1]["w"])
    ref = [FakeTrainingContext(r, native.MLP_TRAINED) for r in range(world)]
    w = np.zeros(native.MLP_TRAINED, np.float32)
    for batches in training.minibatch_schedule(2, 5, 2, 2, 9):
        for slot, s0, s1 in batches:
            g = sum((w - c.target(c.rank, slot, s0)) for c in ref) * np.float32(1.0 / world)
            w = (w - np.float32(0.5) * g.astype(np.float32)).astype(np.float32)
    assert np.allclose(res[0]["w"], w, rtol=1e-6, atol=1e-7)
    sums, count = res[0]["moments"]
    assert count == 30 and np.allclose(sums, np.arange(38) * 3)


class FakeEnergyContext(FakeTrainingContext):
    """The energy-norm step's parts (cs_mlp_energy_begin / _gradient_device / _end) on a vector
    of parameters: the gradient of minibatch [s0, s1) at step k is w - target, the target
    depending on the rank, the step and s0; begin and end count the steps."""

    def __init__(self, rank, n):
        super().__init__(rank, n)
        self.k = 0
        self.open = False

    def mlp_energy_begin(self, params):
        assert not self.open
        self.open = True

    def mlp_energy_gradient_device(self, s0, s1, grad):
        assert self.open
        g = self.w - self.target(self.rank, self.k, s0)
        grad.numpy()[:] = g
        return float(0.5 * (g * g).sum())

    def mlp_energy_end(self, allow_unconverged=False):
        assert self.open
        self.open = False
        self.k += 1
        return None


def _energy_dp_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    from clothsimulator_b200 import native, training

    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    ctx = FakeEnergyContext(rank, native.MLP_TRAINED)
    for step in range(3):
        training.energy_step_data_parallel(ctx, None, 5, 0.5, 2, 40 + step, allreduce_sum=dist.all_reduce,
                                           world=world)
    out[rank] = {"w": ctx.w.copy(), "steps": ctx.k}
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_energy_data_parallel_step_two_gloo_ranks():
    """energy_step_data_parallel over two gloo ranks: identical parameters on both, equal to
    serial descent on the gradients averaged over the ranks, in cs_mlp_train_step's minibatch
    order (its seeded shuffle), each step opened and closed once."""
    sys.path.insert(0, ROOT)
    from clothsimulator_b200 import native, training

    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_energy_dp_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        res = dict(out)
    assert np.array_equal(res[0]["w"], res[1]["w"]) and res[0]["steps"] == 3
    ref = [FakeEnergyContext(r, native.MLP_TRAINED) for r in range(world)]
    w = np.zeros(native.MLP_TRAINED, np.float32)
    for step in range(3):
        (batches,) = list(training.minibatch_schedule(1, 5, 2, 1, 40 + step))
        for _, s0, s1 in batches:
            g = sum((w - c.target(c.rank, step, s0)) for c in ref) * np.float32(1.0 / world)
            w = (w - np.float32(0.5) * g.astype(np.float32)).astype(np.float32)
    assert np.allclose(res[0]["w"], w, rtol=1e-6, atol=1e-7)


# Strong scaling (one workload split across ranks): the sheet partition balanced by stored
# blocks, and the per-sheet statistics gathered back in workload order with one all-gather.

def test_partition_balances_uneven_sheets():
    sys.path.insert(0, ROOT)
    from clothsimulator_b200 import partition, scenes

    scene = scenes.uneven_batch(64, seed=5)
    b = partition.sheet_blocks(scene.sheets)
    for world in (1, 2, 3, 4, 8):
        parts = partition.partition_sheets(b, world)
        got = np.sort(np.concatenate(parts))
        assert np.array_equal(got, np.arange(len(scene.sheets)))  # every sheet exactly once
        # greedy largest-first: within the largest sheet of the mean load
        loads = [int(b[p].sum()) for p in parts]
        assert max(loads) - b.sum() / world <= b.max()
    assert partition.imbalance(b, partition.partition_sheets(b, 4)) < 1.05


def _gather_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    from clothsimulator_b200 import partition

    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(11)
    n = 37
    blocks = rng.integers(100, 5000, n)
    # the statistics a one-rank run would report for every sheet
    full = {"iters": rng.integers(10, 400, n), "rel_residual": rng.uniform(1e-8, 1e-6, n),
            "flags": rng.integers(0, 16, n)}
    parts = partition.partition_sheets(blocks, world)
    mine = parts[rank]
    local = {k: v[mine] for k, v in full.items()}
    got = partition.gather_stats(local, parts, n, partition.torch_all_gather(dist))
    out[rank] = {k: (np.array_equal(got[k], full[k])) for k in full}
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_gathered_stats_equal_one_rank_run_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        assert all(out[r].values()), out[r]
