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
