"""Sheets of one workload split across ranks (one process per GPU), and the per-sheet solver
statistics gathered back in the workload's sheet order.

The reference steps the cloths of a scene one after another (Simulator::physicsStep,
Simulator.cu:584-585); the sheets are independent, so a workload's sheets can be divided among
GPUs with no exchange during the solve.  The cost of a sheet's solve grows with its system's
size, so the split balances the stored 3x3 blocks (nnzb) per rank: greedy largest-first
(each sheet, largest first, to the rank with the fewest blocks so far; ties to the lower rank),
which is within 4/3 of the best split.  After each step the ranks exchange the per-sheet
statistics (CG iterations, final FP64 relative residual, flags) with one all-gather, so every
rank sees the whole workload's convergence.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def sheet_blocks(sheets: Sequence[dict]) -> np.ndarray:
    """Stored 3x3 blocks of each sheet's system, from its triangles alone: the diagonal, and
    both directions of every coupled node pair -- the nodes of a mesh edge, and the two nodes
    opposite an interior edge (bending couples them).  The cost measure the split balances."""
    out = np.zeros(len(sheets), np.int64)
    for k, s in enumerate(sheets):
        f = np.asarray(s["fx"], np.int64)
        n = int(np.asarray(s["x"]).shape[0])
        # every (edge, opposite node) of every face
        e = np.concatenate([f[:, [0, 1, 2]], f[:, [1, 2, 0]], f[:, [2, 0, 1]]])
        lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
        key = lo * n + hi
        order = np.argsort(key, kind="stable")
        key, opp = key[order], e[order, 2]
        edges = np.unique(key)
        # interior edges: a key seen twice; their two opposite nodes are coupled
        twice = np.nonzero(key[1:] == key[:-1])[0]
        a, b = opp[twice], opp[twice + 1]
        pairs = np.unique(np.concatenate([edges, np.minimum(a, b) * n + np.maximum(a, b)]))
        out[k] = n + 2 * len(pairs)
    return out


def partition_sheets(blocks: Sequence[int], world: int) -> list[np.ndarray]:
    """Greedy largest-first split of sheets over `world` ranks balancing the sum of `blocks`.
    Returns, per rank, the indices of its sheets in ascending order."""
    if world < 1:
        raise ValueError("world must be at least 1")
    b = np.asarray(blocks, np.int64)
    order = sorted(range(len(b)), key=lambda i: (-int(b[i]), i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(b[i])
    return [np.array(sorted(p), np.int64) for p in parts]


def imbalance(blocks: Sequence[int], parts: Sequence[np.ndarray]) -> float:
    """Largest rank load over the mean load (1.0 = perfect balance)."""
    b = np.asarray(blocks, np.int64)
    loads = np.array([int(b[p].sum()) for p in parts], np.float64)
    return float(loads.max() / max(loads.mean(), 1.0))


def gather_stats(local: dict, parts: Sequence[np.ndarray], n_sheets: int,
                 all_gather: Callable[[np.ndarray, int], np.ndarray]) -> dict:
    """The whole workload's per-sheet statistics from every rank's own.

    local: this rank's arrays "iters" (int), "rel_residual" (float64), "flags" (int), one entry
    per sheet of its part, in its part's order.  all_gather(buf, count) returns the
    concatenation over ranks of each rank's float64 `buf` padded to `count` rows (one collective;
    NCCL on the device or gloo on the host).  Returns the three arrays in workload sheet order."""
    width = max(len(p) for p in parts)
    buf = np.full((width, 3), np.nan, np.float64)
    k = len(local["iters"])
    buf[:k, 0] = local["iters"]
    buf[:k, 1] = local["rel_residual"]
    buf[:k, 2] = local["flags"]
    allb = np.asarray(all_gather(buf, width)).reshape(len(parts), width, 3)
    out = {"iters": np.zeros(n_sheets, np.int64), "rel_residual": np.zeros(n_sheets, np.float64),
           "flags": np.zeros(n_sheets, np.int64)}
    for r, p in enumerate(parts):
        rows = allb[r, :len(p)]
        out["iters"][p] = rows[:, 0].astype(np.int64)
        out["rel_residual"][p] = rows[:, 1]
        out["flags"][p] = rows[:, 2].astype(np.int64)
    return out


def torch_all_gather(dist, group=None, device=None) -> Callable[[np.ndarray, int], np.ndarray]:
    """An all_gather for gather_stats over a torch.distributed group: the buffer goes to
    `device` (a CUDA device for NCCL, None for gloo on the host), one all_gather."""
    import torch

    def fn(buf: np.ndarray, count: int) -> np.ndarray:
        world = dist.get_world_size(group)
        t = torch.from_numpy(np.ascontiguousarray(buf, np.float64))
        if device is not None:
            t = t.to(device)
        outs = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(outs, t, group=group)
        return torch.cat(outs).cpu().numpy()

    return fn
