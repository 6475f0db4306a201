"""Training of the learned warm start: on one context, or data-parallel over ranks.

`energy_step_data_parallel` is the data-parallel form of cs_mlp_train_step (energy-norm
training along the solver's own trajectories), with the same minibatch order.

cs_mlp_train runs Adam over minibatches of whole sheets of the recorded trajectories on one
GPU.  `train_data_parallel` runs the same schedule on every rank of a process group, each rank
on its own trajectories: the normalisation comes from the moments summed over ranks, and every
minibatch's gradient (a device buffer) is summed over ranks and averaged before the common Adam
step, so all ranks hold the same weights throughout.  With one rank (an identity all-reduce)
it reproduces cs_mlp_train's weights bit for bit: the same minibatch order (the library's
splitmix64 shuffle), gradient kernels and Adam update.
"""
from __future__ import annotations

from typing import Callable

MASK64 = (1 << 64) - 1


def splitmix64(state: int) -> tuple[int, int]:
    """(value, next state) of the splitmix64 generator cs_mlp_train shuffles with."""
    state = (state + 0x9E3779B97F4A7C15) & MASK64
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31), state


def minibatch_schedule(n_slots: int, n_sheets: int, sheets_per_batch: int, epochs: int, seed: int):
    """Per epoch, the (slot, first sheet, end sheet) minibatches in cs_mlp_train's order."""
    groups = (n_sheets + sheets_per_batch - 1) // sheets_per_batch
    order = [(sl, g) for sl in range(n_slots) for g in range(groups)]
    state = seed & MASK64
    for _ in range(epochs):
        for i in range(len(order), 1, -1):
            r, state = splitmix64(state)
            j = r % i
            order[i - 1], order[j] = order[j], order[i - 1]
        yield [(sl, g * sheets_per_batch, min(n_sheets, (g + 1) * sheets_per_batch)) for sl, g in order]


def train_data_parallel(ctx, n_slots: int, n_sheets: int, epochs: int, lr: float, sheets_per_batch: int, seed: int,
                        allreduce_sum: Callable, world: int, sum_host: Callable | None = None) -> list:
    """Adam over this rank's recorded slots with gradients averaged over the group.

    ctx           a native.Context (or an object with its mlp_* methods) whose dataset holds
                  n_slots recorded steps of n_sheets sheets; the weights must start equal on
                  every rank (the same cs_mlp_init seed);
    allreduce_sum sums a CUDA tensor in place over the ranks (e.g. an NCCL all_reduce);
    sum_host      sums a float64 numpy array over the ranks (the normalisation moments);
                  None with one rank.
    Every rank runs the same number of minibatches, so the collectives pair up.  Returns the
    mean minibatch loss per epoch (this rank's data).
    """
    import numpy as np
    import torch

    sums, count = ctx.mlp_moments(n_slots)
    if sum_host is not None:
        both = sum_host(np.concatenate([sums, [float(count)]]))
        sums, count = both[:38], int(round(both[38]))
    ctx.mlp_set_moments(sums, count)
    from .native import MLP_TRAINED

    grad = torch.empty(MLP_TRAINED, dtype=torch.float32, device=ctx.torch_device)
    scale = 1.0 / world
    losses = []
    for batches in minibatch_schedule(n_slots, n_sheets, sheets_per_batch, epochs, seed):
        acc = 0.0
        for slot, s0, s1 in batches:
            acc += ctx.mlp_gradient_device(slot, s0, s1, grad)
            if world > 1:
                allreduce_sum(grad)
                grad.mul_(scale)
                if grad.is_cuda:  # the context's stream reads it next
                    torch.cuda.current_stream(grad.device).synchronize()
            ctx.mlp_apply_gradient(grad, lr)
        losses.append(acc / max(len(batches), 1))
    return losses


def energy_step_data_parallel(ctx, params, n_sheets: int, lr: float, sheets_per_batch: int, seed: int,
                              allreduce_sum: Callable, world: int, grad=None, allow_unconverged: bool = True):
    """One step of energy-norm training (cs_mlp_train_step) with gradients averaged over the
    group: this rank's step is solved and updated as cs_mlp_train_step does it, and every
    minibatch of cs_mlp_train_step's order (its seeded shuffle) takes the Adam step on the
    gradient summed over the ranks and divided by their number.  Every rank has the same
    number of sheets, so the collectives pair up.  Returns (step statistics, mean minibatch
    loss of this rank)."""
    import torch

    from .native import MLP_TRAINED

    if grad is None:
        grad = torch.empty(MLP_TRAINED, dtype=torch.float32, device=ctx.torch_device)
    ctx.mlp_energy_begin(params)
    (batches,) = list(minibatch_schedule(1, n_sheets, sheets_per_batch, 1, seed))
    acc = 0.0
    for _, s0, s1 in batches:
        acc += ctx.mlp_energy_gradient_device(s0, s1, grad)
        if world > 1:
            allreduce_sum(grad)
            grad.mul_(1.0 / world)
            if grad.is_cuda:
                torch.cuda.current_stream(grad.device).synchronize()
        ctx.mlp_apply_gradient(grad, lr)
    stats = ctx.mlp_energy_end(allow_unconverged=allow_unconverged)
    return stats, acc / max(len(batches), 1)
