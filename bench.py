"""Benchmark of the implicit cloth step on B200.

Workloads (--workload; the default is the headline):
  windy1024x64   1,024 sheets of 64x64 quads (4,326,400 nodes), top edge pinned, per-sheet
                 horizontal wind, stretching log-U[10, 500] N/m and bending log-U[1e-6, 1e-3] N m
                 through the material multipliers, dt = 1/100 s: the learned-warm-start
                 configuration, the largest that fits one GPU, and the one the metric is quoted on;
  hang32         one 32x32 hanging sheet, 200 steps;
  precision256   one 256x256 sheet, one step, solved to 1e-6 (mixed and plain FP32) and 1e-10;
  uneven512      512 sheets of 16..128 quads a side, 1-4 corners pinned, 100 steps;
  irregular1000  one 1,000x1,000 jittered sheet with random diagonals (1,002,001 nodes), wind,
                 50 steps, the windy network as warm start.
One step = assembly + PCG to an FP64-checked relative residual of 1e-6 for every sheet +
v += dv, x += dt v, with the state resident in HBM.

Metric: node-steps/s (sum over sheets of nodes x steps / device time).  The line reports the
mixed-precision solver (`value`: cluster-resident solve where a sheet fits, strip-local Chebyshev
preconditioner of degree --precond-degree with the coarse-space correction, reliable updates; the
workload's warm start) and, in `arms`, the same solver without the coarse correction, with
block-Jacobi, from other starts, at the tolerance that meets the dv bound, and plain FP32 PCG from
a zero guess on the same GPU, each with its dv error against an FP64 solve of its own system on
sampled sheets.  `--impl reference` times the reference's CPU path for the workload (the
reference's own force code compiled from its sources + FP32 sparse Cholesky).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload W]
       torchrun --nproc-per-node N bench.py --gpus N [--partition]
         (one rank per GPU; each rank its own copy of the workload (weak scaling), or with
          --partition one workload's sheets split across the ranks (strong scaling))
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s @ rel.res 1e-6: learned+mixed-prec batched PCG vs plain FP32 PCG"
UNIT = "node-steps/s"


WORKLOADS = ("windy1024x64", "hang32", "precision256", "uneven512", "irregular1000")


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default: 10, or the workload's own "
                    "step count when it is smaller than 10 seconds of work: hang32 200, uneven512 100, "
                    "irregular1000 50, precision256 1)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="windy1024x64", choices=WORKLOADS)
    ap.add_argument("--sheets", type=int, default=None, help="windy workload: sheets (default 1,024)")
    ap.add_argument("--nq", type=int, default=64, help="windy workload: quads per side")
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--dv-tol", type=float, default=1e-7,
                    help="the tolerance of the arm that meets the dv bound of 1e-6 against an FP64 solve")
    ap.add_argument("--warm", default=None, choices=["previous", "zero", "learned"],
                    help="the warm start of the headline arm (default: learned for the windy and irregular "
                         "workloads, previous dv for the others)")
    ap.add_argument("--solver", default="auto", choices=["auto", "batched"],
                    help="auto: sheets that fit a cluster's shared memory are solved cluster-resident")
    ap.add_argument("--precond-degree", type=int, default=3,
                    help="cluster-resident solver's preconditioner: 1 block-Jacobi, odd 3..15 a strip-local "
                         "Chebyshev polynomial of that degree (the batched loop always uses block-Jacobi)")
    ap.add_argument("--no-coarse", action="store_true", help="headline arm without the coarse-space correction")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (cs_tune)")
    ap.add_argument("--fixed-precond", action="store_true",
                    help="keep --precond-degree / --no-coarse for the headline instead of the tuner's choice")
    ap.add_argument("--partition", action="store_true",
                    help="with several ranks: split one workload's sheets across them, balanced by stored blocks "
                         "(strong scaling), per-sheet statistics all-gathered after each step")
    ap.add_argument("--train-loss", default="energy", choices=["energy", "mse"],
                    help="energy: online training on the trajectories' own systems, loss = relative error of the "
                         "prediction in the energy norm (cs_mlp_train_step); mse: recorded (state, dv) pairs, "
                         "squared error of dv (cs_mlp_train)")
    ap.add_argument("--train-sheets", type=int, default=None,
                    help="sheets (trajectories) of the training set (default: energy 1,024, mse 256)")
    ap.add_argument("--train-steps", type=int, default=None,
                    help="steps per training trajectory (default: energy 200, mse 24)")
    ap.add_argument("--epochs", type=int, default=None, help="passes over the trajectories (default: energy 1, mse 16)")
    ap.add_argument("--train-lr", type=float, default=1e-3)
    ap.add_argument("--train-batch", type=int, default=16, help="sheets per minibatch (energy training)")
    ap.add_argument("--weights", default="", help="load trained warm-start weights instead of training")
    ap.add_argument("--no-plain", action="store_true", help="skip the comparison arms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-dv-check", action="store_true", help="skip the dv errors of the arms")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--detect", default="", choices=["", "windy", "stacked", "folded", "crossing"],
                    help="time proximity detection, the step and the collision step on a contact workload "
                         "instead: windy = the 1,024-sheet batch, a group per sheet; stacked = two 256x256 "
                         "sheets 1.5 mm apart; folded = one 256x256 sheet folded onto itself; crossing = "
                         "stacked with the upper sheet moving down at 0.5 m/s")
    ap.add_argument("--host-loop", action="store_true",
                    help="launch the solve loop from the host instead of the CUDA graph (profilers cannot "
                         "see kernels inside a graph with conditional nodes)")
    args = ap.parse_args(argv)
    spec = workload_spec(args.workload)
    if args.steps is None:
        args.steps = spec["steps"]
    if args.warm is None:
        args.warm = spec["warm"]
    if args.sheets is None:
        args.sheets = 1024
    return args


def workload_spec(name: str) -> dict:
    """Timed steps by default, the headline arm's warm start, and whether the workload is one
    sheet (its CPU baseline then times a smaller instance of the same scene)."""
    return {
        "windy1024x64": {"steps": 10, "warm": "learned", "single": False},
        "hang32": {"steps": 200, "warm": "previous", "single": True},
        "precision256": {"steps": 1, "warm": "zero", "single": True},
        "uneven512": {"steps": 100, "warm": "previous", "single": False},
        "irregular1000": {"steps": 50, "warm": "learned", "single": True},
    }[name]


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class RankGroup:
    """One process per GPU (torchrun).  Sheets are independent, so ranks exchange no data during
    the solve: the group carries the barriers around the timed region and the max over ranks of
    the device times (gloo, host scalars); an NCCL group beside it carries the warm start's
    gradient all-reduce and, with --partition, the all-gather of the per-sheet statistics."""

    def __init__(self, timeout_s: float = 300.0):
        import datetime

        self.rank, self.world, self.local = dist_env()
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.dist:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_host(self, a):
        """Sum of a float64 numpy array over the ranks (gloo)."""
        if not self.dist:
            return a
        import torch

        t = torch.from_numpy(np.array(a, np.float64))
        self.dist.all_reduce(t)
        return t.numpy()

    def nccl_group(self):
        """An NCCL group of all ranks beside the gloo group of the host scalars (created once)."""
        if not self.dist:
            return None
        if getattr(self, "_nccl", None) is None:
            self._nccl = self.dist.new_group(backend="nccl")
        return self._nccl

    def device_allreduce(self):
        """An in-place sum of CUDA tensors over the ranks: NCCL over NVLink (a group of its own
        beside the gloo group of the host scalars)."""
        if not self.dist:
            return None
        grp = self.nccl_group()
        return lambda t: self.dist.all_reduce(t, group=grp)

    def close(self):
        if self.dist:
            if getattr(self, "_nccl", None) is not None:
                self.dist.destroy_process_group(self._nccl)
                self._nccl = None
            self.dist.destroy_process_group()
            self.dist = None


def eval_seed(rank: int) -> int:
    """Seed of the evaluated workload of a rank."""
    return 1000 + rank


def train_seed(rank: int) -> int:
    """Seed of a rank's warm-start training trajectories: disjoint from every evaluated seed
    for up to 32 ranks (7 + 31 r < 1000)."""
    return 7 + 31 * rank


def aggregate_value(nodes_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job node-steps/s: every rank steps its own batch; time = the slowest rank's."""
    return nodes_per_rank * steps * world / (ms_max / 1e3)


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [t.strip() for t in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except FileNotFoundError:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def scenes_mod():
    from clothsimulator_b200 import scenes

    return scenes


def workload(args, rank, small: bool = False):
    """The scene a rank steps (each rank its own seed: weak scaling).  small=True: a smaller
    instance of a single-sheet scene for the CPU baseline's bounded sample."""
    sc = scenes_mod()
    seed = eval_seed(rank)
    if args.workload == "windy1024x64":
        return sc.windy_batch(args.sheets, args.nq, seed=seed)
    if args.workload == "hang32":
        return sc.hang(32, seed=seed)
    if args.workload == "precision256":
        return sc.precision_sheet(128 if small else 256, seed=seed)
    if args.workload == "uneven512":
        return sc.uneven_batch(512, seed=seed)
    return sc.large_irregular(200 if small else 1000, seed=seed)


def cpu_baseline(scene, seconds: float, which: str = "ref", threads: int = 1, n_steps: int = 1):
    """Times the reference CPU path (FP32 assembly + FP32 sparse Cholesky, one sheet after
    another as Simulator.cu:584-585 does) on a bounded sample of the workload's sheets."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from clothsimulator_b200 import scenes

    if which == "ref" and not os.path.exists(pyoracle.LIB_REF):
        which = "oracle"
    kind = "reference" if which == "ref" else "port"
    sheets = scene.sheets
    # calibrate on one sheet (first step includes the symbolic analysis, as SimplicialLLT does)
    mk = (lambda s: pyoracle.Cloth(s, pyoracle.Material(s["material"], which=which))) if which == "ref" else \
        (lambda s: pyoracle.Cloth(s, pyoracle.Material(s["material"], "float")))
    c0 = mk(sheets[0])
    t0 = time.perf_counter()
    c0.step(scenes.step_params(scene, sheets[0]), pyoracle.METHOD_LLT)
    one = max(time.perf_counter() - t0, 1e-4)
    count = int(max(threads, min(len(sheets), math.ceil(seconds * threads / (one * n_steps)))))
    cloths = [mk(s) for s in sheets[:count]]
    params = [scenes.step_params(scene, s) for s in sheets[:count]]
    sec, status = pyoracle.run_cloths(cloths, params, n_steps, pyoracle.METHOD_LLT, threads)
    nodes = sum(s["x"].shape[0] for s in sheets[:count])
    return {
        "value": nodes * n_steps / sec,
        "unit": UNIT,
        "cores": threads,
        "kind": kind,
        "sample": f"{count} of {len(sheets)} sheets ({scene.name}), {n_steps} step(s) each, "
                  f"{'reference force code' if kind == 'reference' else 'restated force code'} + FP32 sparse LL^T, "
                  f"{sec:.1f} s on {threads} thread(s)",
        "failed_solves": int((status < -1).sum()),
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    scene = workload(args, 0, small=workload_spec(args.workload)["single"])
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(1, args.warmup)):
        cpu_baseline(scene, 2.0, "ref", threads)
    samples = []
    for _ in range(args.steps):
        r = cpu_baseline(scene, max(0.2, 4.0 * args.cpu_seconds / max(1, args.steps)), "ref", threads)
        vals.append(r["value"])
        samples.append(r["sample"])
    value = statistics.median(vals)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "sheets": len(workload_sheets(args)), "tol": args.tol},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": r["kind"], "sample": samples[-1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def workload_sheets(args):
    """The sheets of the workload at full size (the reference arm's config names them)."""
    return workload(args, 0).sheets


def train_warm_start(args, group, local):
    """The learned warm start: trained on the device on separate seeded windy trajectories (the
    evaluated seeds are held out), or loaded from --weights.  Returns (weights, training record).

    energy (default): the network is trained online along 1,024 trajectories of 200 steps (the
    specified training set), each step solved by the solver without the learned start; between
    a step's solve and its state update, one Adam step per minibatch of sheets on the energy-norm
    loss of the prediction for that step's system (cs_mlp_train_step), the normalisation fitted
    first on a few recorded steps.  mse: recorded (state, dv) pairs, squared error
    (cs_mlp_train).  With several ranks both train data parallel: each rank on its own
    trajectories, gradients averaged over NCCL."""
    from clothsimulator_b200 import native

    rank, world = group.rank, group.world
    t0 = time.perf_counter()
    energy = args.train_loss == "energy"
    sheets = args.train_sheets or (1024 if energy else 256)
    steps = args.train_steps or (200 if energy else 24)
    epochs = args.epochs or (1 if energy else 16)
    if args.weights:
        weights = np.fromfile(args.weights, dtype=np.float32)
        info = {"source": args.weights}
    elif energy:
        tscene = scenes_mod().windy_batch(sheets, args.nq, seed=train_seed(rank))
        tctx = native.Context(local)
        tctx.load(tscene.sheets)
        n_norm = 6
        tctx.mlp_init(n_norm, 1)  # the same initial weights on every rank
        tp = native.step_params(tscene.dt, tscene.gravity, tscene.handle_stiffness, tol=args.tol, max_iters=20000,
                                precond_degree=3, coarse=1)
        # normalisation from the features and targets of steps 10-15 (past the start from rest;
        # moments summed over the ranks); the output is not shifted (mean 0, scale the targets'
        # RMS), so that the untrained network predicts about the previous dv
        n_skip = 10
        for t in range(n_skip + n_norm):
            if t >= n_skip:
                tctx.assemble(tp)
                tctx.mlp_record(t - n_skip, 0)
            tctx.step(tp, allow_unconverged=True)
            if t >= n_skip:
                tctx.mlp_record(t - n_skip, 1)
            tp.warm_start = native.WARM_PREVIOUS
        sums, count = tctx.mlp_moments(n_norm)
        if world > 1:
            both = group.sum_host(np.concatenate([sums, [float(count)]]))
            sums, count = both[:38], int(round(both[38]))
        sums[16:19] = 0.0
        tctx.mlp_set_moments(sums, count)
        xs = np.concatenate([s["x"] for s in tscene.sheets])
        vs = np.concatenate([s["v"] for s in tscene.sheets])
        curve = []
        if world > 1:
            # data parallel: every rank steps its own trajectories, each minibatch's gradient
            # summed over NCCL and averaged before the common Adam step
            import torch

            from clothsimulator_b200 import training

            grad = torch.empty(native.MLP_TRAINED, dtype=torch.float32, device=torch.device("cuda", local))
            allreduce = group.device_allreduce()
        for ep in range(epochs):
            tctx.set_state(xs, vs)
            tp.warm_start = native.WARM_ZERO
            ep_loss = []
            for t in range(steps):
                seed = 1 + ep * steps + t
                if t < 2:
                    # the first steps from rest (no previous dv yet) are not trained on
                    tctx.step(tp, allow_unconverged=True)
                elif world > 1:
                    _, loss = training.energy_step_data_parallel(tctx, tp, sheets, args.train_lr, args.train_batch, seed,
                                                                 allreduce, world, grad=grad)
                    ep_loss.append(loss)
                else:
                    _, loss = tctx.mlp_train_step(tp, lr=args.train_lr, sheets_per_batch=args.train_batch, seed=seed,
                                                  allow_unconverged=True)
                    ep_loss.append(loss)
                tp.warm_start = native.WARM_PREVIOUS
            curve.append(ep_loss)
        weights = tctx.mlp_get_weights()
        tctx.close()
        first, last = curve[0], curve[-1]
        k = max(1, len(first) // 10)
        info = {"loss": "sin^2 of the angle between prediction and solution in the energy inner product of the "
                        "step's system (the Galerkin-scaled start's squared energy error relative to the zero "
                        "guess's), mean over sheets",
                "sheets": sheets, "steps": steps, "epochs": epochs, "lr": args.train_lr,
                "sheets_per_minibatch": args.train_batch,
                "adam_steps": epochs * (steps - 2) * ((sheets + args.train_batch - 1) // args.train_batch),
                "trajectories": f"windy{sheets}x{args.nq} per rank, seeds disjoint from the evaluated workload, "
                                "solved without the learned start (mixed PCG, Chebyshev-3 + coarse correction)",
                "loss_first_steps": float(np.mean(first[:k])), "loss_last_steps": float(np.mean(last[-k:])),
                "loss_epoch_means": [float(np.mean(c)) for c in curve]}
        if world > 1:
            digest = float(np.float64(weights).sum())
            info["data_parallel"] = {"ranks": world, "gradients": "NCCL all-reduce, averaged",
                                     "weights_identical": group.max(digest) == -group.max(-digest)}
    else:
        tscene = scenes_mod().windy_batch(sheets, args.nq, seed=train_seed(rank))
        tctx = native.Context(local)
        tctx.load(tscene.sheets)
        tctx.mlp_init(steps, 1)  # the same initial weights on every rank
        tp = native.step_params(tscene.dt, tscene.gravity, tscene.handle_stiffness, tol=1e-7, max_iters=8000)
        for _ in range(2):
            tctx.step(tp, allow_unconverged=True)
            tp.warm_start = native.WARM_PREVIOUS
        for t in range(steps):
            tctx.assemble(tp)
            tctx.mlp_record(t, 0)
            tctx.step(tp, allow_unconverged=True)
            tctx.mlp_record(t, 1)
        if world == 1:
            tctx.mlp_fit_normalization(steps)
            losses = tctx.mlp_train(steps, epochs, lr=args.train_lr, sheets_per_batch=32, seed=3)
        else:
            # data parallel: every rank trains on its own trajectories, gradients summed over
            # NCCL and averaged, normalisation from the moments summed over the ranks
            from clothsimulator_b200 import training

            losses = training.train_data_parallel(tctx, steps, sheets, epochs, args.train_lr,
                                                  32, 3, allreduce_sum=group.device_allreduce(), world=world,
                                                  sum_host=group.sum_host)
        weights = tctx.mlp_get_weights()
        tctx.close()
        info = {"loss": "squared error of dv", "sheets": sheets, "steps": steps, "epochs": epochs,
                "trajectories": f"windy{sheets}x{args.nq}, seeds disjoint from the evaluated workload",
                "loss_first": float(losses[0]), "loss_last": float(losses[-1])}
        if world > 1:
            digest = float(np.float64(weights).sum())
            info["data_parallel"] = {"ranks": world, "gradients": "NCCL all-reduce, averaged",
                                     "weights_identical": group.max(digest) == -group.max(-digest)}
    info["seconds"] = time.perf_counter() - t0
    return weights, info


def dv_errors(sheets, scene, local, params, weights=None, n_sample=8):
    """dv error of one solver arm: max over a seeded sample of the sheets of
    ||dv - dv_64|| / ||dv_64||, where dv_64 is an FP64 direct solve (SciPy) of the system the GPU
    assembled for that sheet, one step from the sheet's initial state (a context of its own with
    the sampled sheets; the sheets are independent, so their systems are the same as in the
    whole batch)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl

    from clothsimulator_b200 import native

    rng = np.random.default_rng(5)
    pick = sorted(rng.choice(len(sheets), min(n_sample, len(sheets)), replace=False).tolist())
    sub = [sheets[k] for k in pick]
    ctx = native.Context(local).load(sub)
    if weights is not None:
        ctx.mlp_init(0, 0)
        ctx.mlp_set_weights(weights)
    x0 = np.concatenate([s["x"] for s in sub])
    v0 = np.concatenate([s["v"] for s in sub])
    p = native.StepParams.from_buffer_copy(params)
    p.advance = 0
    if p.warm_start == native.WARM_PREVIOUS:
        p.warm_start = native.WARM_ZERO  # one step from the initial state: no previous dv
    ctx.set_state(x0, v0)
    ctx.step(p, allow_unconverged=True)
    dv = ctx.get_dv().reshape(-1)
    ctx.assemble(p)
    rp, ci, val, b = ctx.system()
    errs, off = [], 0
    for s in sub:
        n = s["x"].shape[0]
        lo, hi = int(rp[off]), int(rp[off + n])
        A = sp.bsr_matrix((val[lo:hi].astype(np.float64), (ci[lo:hi] - off).astype(np.int64),
                           (rp[off:off + n + 1] - lo).astype(np.int64)), shape=(3 * n, 3 * n)).tocsc()
        exact = spl.spsolve(A, b[3 * off:3 * (off + n)].astype(np.float64))
        d = dv[3 * off:3 * (off + n)].astype(np.float64)
        errs.append(float(np.linalg.norm(d - exact) / np.linalg.norm(exact)))
        off += n
    ctx.close()
    e = np.array(errs)
    return {"dv_err_vs_fp64": float(np.max(e)) if np.all(np.isfinite(e)) else None,
            "dv_err_sheets": len(sub), "dv_err_all_finite": bool(np.all(np.isfinite(e)))}


def run_ours(args):
    import torch

    from clothsimulator_b200 import native, partition

    group = RankGroup()
    rank, world, local = group.rank, group.world, group.local
    torch.cuda.set_device(local)
    spec = workload_spec(args.workload)
    if args.partition and world > 1:
        # strong scaling: one workload (rank 0's seed), its sheets split across the ranks
        full = workload(args, 0)
        blocks = partition.sheet_blocks(full.sheets)
        parts = partition.partition_sheets(blocks, world)
        scene = scenes_mod().Scene(full.name, [full.sheets[k] for k in parts[rank]], dt=full.dt, steps=full.steps,
                                   gravity=full.gravity, handle_stiffness=full.handle_stiffness)
        part_info = {"ranks": world, "sheets_per_rank": [len(p) for p in parts],
                     "blocks_imbalance": partition.imbalance(blocks, parts)}
    else:
        scene = workload(args, rank)
        parts, part_info = None, None
    ctx = native.Context(local)
    ctx.load(scene.sheets)
    sizes = ctx.sizes
    N = sizes[0]
    total_nodes = int(group.sum_host(np.array([float(N)]))[0])
    x0 = np.concatenate([s["x"] for s in scene.sheets])
    v0 = np.concatenate([s["v"] for s in scene.sheets])
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))
    barrier = group.barrier
    max_over_ranks = group.max

    # autotuner: the batched SpMV's launch shape (applied from now on) and the fastest resident
    # preconditioner, timed on this batch (cs_tune) at the state the timed steps start from
    # (after the warm-up steps; the first step from rest is dominated by the near-rigid
    # gravity/wind mode, which the coarse correction alone resolves in a few iterations)
    tuning = None
    if not args.no_tune:
        tp = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol, max_iters=20000,
                                precond_degree=args.precond_degree)
        ctx.set_state(x0, v0)
        for _ in range(args.warmup):
            ctx.step(tp, allow_unconverged=True)
        t = ctx.tune(tp, reps=5)
        default = next(x for x in t["spmv"] if (x["threads"], x["slices_per_warp"], x["unroll"]) == (128, 1, 1))
        tuning = {"spmv": {k: t["spmv"][t["best_spmv"]][k] for k in ("threads", "slices_per_warp", "unroll", "ms")},
                  "spmv_default_ms": default["ms"], "spmv_shapes_identical_bits": len({x["checksum"] for x in t["spmv"]}) == 1,
                  "precond": t["precond"][t["best_precond"]] if t["best_precond"] >= 0 else None,
                  "precond_candidates": t["precond"]}
        tuning["solver_ms"] = t["solver_ms"]
        tuning["solver"] = t["best_solver"]
        if t["best_precond"] >= 0 and not args.fixed_precond:
            args.precond_degree = t["precond"][t["best_precond"]]["degree"]
            args.no_coarse = not t["precond"][t["best_precond"]]["coarse"]
        if args.solver == "auto" and t["best_solver"] == "batched" and not args.fixed_precond:
            args.solver = "batched"

    weights, train_info = None, None
    if args.warm == "learned":
        weights, train_info = train_warm_start(args, group, local)
        ctx.mlp_init(0, 0)
        ctx.mlp_set_weights(weights)
        if all(s["x"].shape[0] <= 300000 for s in scene.sheets) and not any(len(s.get("prox", [])) for s in scene.sheets):
            # the energy-norm loss (sin^2 of the A-angle to the solution; the Galerkin-scaled
            # start's squared energy error relative to the zero guess's) on this workload at the
            # state the timed steps start from, for the trained network and for the previous dv
            # alone (the network with its output layer zeroed)
            ep = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol, max_iters=20000,
                                    precond_degree=3, coarse=1, warm_start=native.WARM_PREVIOUS, advance=0)
            _, l_net = ctx.mlp_energy_gradient(ep, 0, ctx.n_sheets)
            w0 = np.array(weights, np.float32)
            w0[14528:native.MLP_TRAINED] = 0.0  # output layer W4, b4
            ctx.mlp_set_weights(w0)
            _, l_prev = ctx.mlp_energy_gradient(ep, 0, ctx.n_sheets)
            ctx.mlp_set_weights(weights)
            train_info["evaluated_sin2"] = {"network": l_net, "previous_dv": l_prev,
                                            "state": "the evaluated workload after the warm-up steps"}

    solver_code = {"auto": native.SOLVER_AUTO, "batched": native.SOLVER_BATCHED}
    warm_code = {"previous": native.WARM_PREVIOUS, "zero": native.WARM_ZERO, "learned": native.WARM_LEARNED}

    def arm_params(precision, solver, degree, coarse, tol):
        return native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=tol, max_iters=20000,
                                  precision=precision, warm_start=native.WARM_ZERO,
                                  use_graph=0 if args.host_loop else 1, solver=solver_code[solver],
                                  precond_degree=degree, coarse=coarse)

    def timed_arm(precision, warm, solver, degree, coarse, tol, clocks=None):
        ctx.set_state(x0, v0)
        p = arm_params(precision, solver, degree, coarse, tol)
        # the learned start is replaced by its Galerkin multiple before the guard (warm_scale)
        p.warm_scale = 1 if warm == native.WARM_LEARNED else 0
        for i in range(args.warmup):
            ctx.step(p, allow_unconverged=True)
            p.warm_start = warm
        p.warm_start = warm
        c0 = ctx.counters()
        barrier()
        torch.cuda.synchronize()
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if clocks is not None else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        for i in range(args.steps):
            ctx.step_async(p)
        e1.record(stream)
        e1.synchronize()
        if sampler:
            sampler.__exit__()
            clocks.update(sampler.summary())
        torch.cuda.synchronize()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))
        c1 = ctx.counters()
        # one untimed step with statistics for the report (and, with --partition, the whole
        # workload's per-sheet statistics gathered from every rank)
        ctx.step(p, allow_unconverged=True)
        it, rr, fl = ctx.instance_stats()
        if parts is not None:
            g = partition.gather_stats({"iters": it, "rel_residual": rr, "flags": fl}, parts, sum(len(q) for q in parts),
                                       partition.torch_all_gather(group.dist, group.nccl_group(),
                                                                  torch.device("cuda", local)))
            it, rr, fl = g["iters"], g["rel_residual"], g["flags"]
        return {
            "value": total_nodes * args.steps / (ms / 1e3),
            "ms": ms,
            "ms_per_step": ms / args.steps,
            "launches": c1["launches"] - c0["launches"],
            "iters_mean": float(it.mean()),
            "iters_max": int(it.max()),
            "converged_frac": float(np.mean((fl & 1) > 0)),
            "warm_rejected_frac": float(np.mean((fl & 2) > 0)),
            "max_relres": float(rr.max()),
        }, p

    keys = ("value", "ms_per_step", "iters_mean", "iters_max", "converged_frac", "warm_rejected_frac", "max_relres")
    deg = args.precond_degree
    coarse = 0 if args.no_coarse else 1
    clocks = {}
    best, best_p = timed_arm(native.PREC_MIXED, warm_code[args.warm], args.solver, deg, coarse, args.tol, clocks)
    value = best["value"]
    head = f"mixed_{args.warm}_{args.solver}"
    arms = {head: dict({k: best[k] for k in keys}, precond_degree=deg if args.solver == "auto" else 1,
                       coarse=coarse, tol=args.tol)}
    arm_params_used = {head: best_p}
    if not args.no_plain:
        # the plain FP32 arms keep block-Jacobi and the zero guess (the reference's solver
        # structure); the mixed arms use --precond-degree, without and with the coarse correction,
        # with block-Jacobi beside them, and at --dv-tol (the tolerance whose dv meets 1e-6)
        P, M = native.PREC_PLAIN_FP32, native.PREC_MIXED
        W = warm_code[args.warm]
        cand = [("mixed_zero_auto", M, native.WARM_ZERO, "auto", deg, 1, args.tol),
                ("mixed_previous_auto", M, native.WARM_PREVIOUS, "auto", deg, 1, args.tol),
                (f"mixed_{args.warm}_auto_no_coarse", M, W, "auto", deg, 0, args.tol),
                (f"mixed_{args.warm}_auto_block_jacobi", M, W, "auto", 1, 0, args.tol),
                (f"mixed_{args.warm}_auto_tol{args.dv_tol:g}", M, W, "auto", deg, 1, args.dv_tol),
                ("plain_fp32_zero_auto", P, native.WARM_ZERO, "auto", 1, 0, args.tol),
                ("mixed_previous_batched", M, native.WARM_PREVIOUS, "batched", 1, 0, args.tol),
                ("plain_fp32_zero_batched", P, native.WARM_ZERO, "batched", 1, 0, args.tol)]
        if args.workload == "precision256":
            cand.append(("mixed_zero_auto_tol1e-10", M, native.WARM_ZERO, "auto", deg, 1, 1e-10))
        # the arms each workload reports (a single large sheet is solved by the batched loop,
        # where the preconditioner options do not apply)
        keep = {"windy1024x64": None,
                "uneven512": {"mixed_zero_auto", "no_coarse", "block_jacobi", "tol", "plain_fp32_zero_auto",
                              "plain_fp32_zero_batched", "mixed_previous_batched"},
                "hang32": {"mixed_zero_auto", "no_coarse", "block_jacobi", "plain_fp32_zero_auto"},
                "precision256": {"no_coarse", "plain_fp32_zero_auto", "tol1e-10"},
                "irregular1000": {"mixed_zero_auto", "plain_fp32_zero_batched"}}[args.workload]
        for name, prec, warm, solver, d, co, tol in cand:
            if name in arms or (name.endswith("block_jacobi") and deg == 1):
                continue
            if keep is not None and not any(name == k or name.endswith(k) or f"_{k}" in name for k in keep):
                continue
            r, pr = timed_arm(prec, warm, solver, d, co, tol)
            arms[name] = dict({k: r[k] for k in keys}, precond_degree=d if solver == "auto" else 1, coarse=co, tol=tol)
            arm_params_used[name] = pr
    plain = arms.get("plain_fp32_zero_batched")

    # dv error of every arm against an FP64 solve of its own assembled system (sampled sheets)
    if not args.no_dv_check and rank == 0 and max(s["x"].shape[0] for s in scene.sheets) <= 300000:
        for name, pr in arm_params_used.items():
            use_w = weights if pr.warm_start == native.WARM_LEARNED else None
            arms[name].update(dv_errors(scene.sheets, scene, local, pr, use_w))

    # Rooflines, timed live on the context's stream (cs_profile_kernels).  The dominant kernel
    # of the step (resident solver, when sheets are resident): algorithmic bytes per launch =
    # CG iterations x (stored blocks x 40 B + nodes x 48 B), the per-iteration bytes of a
    # streaming PCG (the same figure as the batched SpMV's); the kernel serves them from
    # shared memory, so `roofline_smem` sets the shared-memory bytes it moves against the
    # shared-memory bandwidth of the SMs it runs on.
    prof = ctx.profile_kernels(arm_params(native.PREC_MIXED, args.solver, deg, coarse, args.tol), reps=3)
    info = ctx.solver_info()
    all_resident = info["resident_sheets"] == len(scene.sheets) and prof["resident_solve"] > 0
    # the per-sheet statistics of the timed resident solve (kept when it solved every sheet)
    it_res = ctx.instance_stats()[0] if all_resident else None
    nnzb = sizes[6]
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    src = "measured" if peaks else "fallback"

    def traffic_per_launch(name, units):
        path = os.path.join(ROOT, "profiles", name)
        if os.path.exists(path):
            t = json.load(open(path))
            if t.get("dram_bytes"):
                return t["dram_bytes"] * units / t[t["per"]]
        return None

    spmv_bytes = nnzb * 40 + N * 48
    spmv_achieved = spmv_bytes / (prof["spmv"] * 1e-3) / 1e9
    roof_spmv = {"bound": "hbm", "achieved": spmv_achieved, "peak": peak, "unit": "GB/s", "frac": spmv_achieved / peak,
                 "traffic": traffic_per_launch("cs_spmv_kernel_windy128x64_traffic.json", N),
                 "kernel": "cs_spmv_kernel", "bytes_per_launch": spmv_bytes, "ms_per_launch": prof["spmv"],
                 "peak_source": src}
    roof_res, roof_smem = None, None
    if all_resident and args.solver == "auto":
        per_sheet = np.array([(s["x"].shape[0]) for s in scene.sheets], np.float64)
        blocks_sheet = partition.sheet_blocks(scene.sheets).astype(np.float64)
        if True:
            res_bytes = float(np.sum(it_res * (blocks_sheet * 40 + per_sheet * 48)))
            ms_res = prof["resident_solve"]
            res_achieved = res_bytes / (ms_res * 1e-3) / 1e9
            roof_res = {"bound": "hbm", "achieved": res_achieved, "peak": peak, "unit": "GB/s",
                        "frac": res_achieved / peak,
                        "traffic": traffic_per_launch("cs_resident_pcg_kernel_windy32x64_traffic.json", len(scene.sheets)),
                        "kernel": "cs_resident_pcg_kernel", "bytes_per_launch": res_bytes, "ms_per_launch": ms_res,
                        "cg_iterations_per_launch": int(it_res.sum()), "peak_source": src,
                        "note": "algorithmic bytes = CG iterations x (stored blocks x 40 B + nodes x 48 B), what a "
                                "streaming PCG would move; the kernel reads them from shared memory (roofline_smem)"}
            # shared-memory bytes: per CG iteration the full SpMV (36 B of block values + 16 B of
            # the vector per stored block) and (degree - 1) strip-local SpMVs over the strip-local
            # blocks; per solve the power iterations
            rb = ctx.resident_blocks()
            local_frac = rb["local_blocks"] / max(rb["blocks"], 1)
            cheb = deg >= 3
            smem_bytes = float(np.sum(it_res * blocks_sheet * 52 * (1 + (deg - 1) * local_frac * cheb)
                                      + cheb * rb["power_iters"] * local_frac * blocks_sheet * 52))
            sm_mhz = clocks.get("sm_mhz") or 1965.0
            sms = info["clusters"] * info["ctas_per_cluster"]
            smem_peak = 128.0 * sms * sm_mhz * 1e6 / 1e9
            smem_achieved = smem_bytes / (ms_res * 1e-3) / 1e9
            roof_smem = {"bound": "smem", "achieved": smem_achieved, "peak": smem_peak, "unit": "GB/s",
                         "frac": smem_achieved / smem_peak, "kernel": "cs_resident_pcg_kernel",
                         "bytes_per_launch": smem_bytes, "sms": sms, "sm_mhz": sm_mhz,
                         "peak_source": "128 B per clock per SM x SMs the kernel runs on x sampled SM clock"}
    roofline = roof_res if roof_res else roof_spmv

    # end to end through the C ABI with pinned host buffers: H2D of x, v, step, D2H of x, v
    node_steps = total_nodes * args.steps
    hx = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
    hv = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
    hx.numpy()[:] = x0
    hv.numpy()[:] = v0
    fp = native._fp
    import ctypes as C

    px = C.cast(hx.data_ptr(), fp)
    pv = C.cast(hv.data_ptr(), fp)
    p = arm_params(native.PREC_MIXED, args.solver, deg, coarse, args.tol)
    ctx.set_state(x0, v0)
    for i in range(args.warmup):
        ctx.check(ctx.lib.cs_set_state(ctx.h, px, pv))
        ctx.step(p, allow_unconverged=True)
        ctx.check(ctx.lib.cs_get_state(ctx.h, px, pv))
        p.warm_start = warm_code[args.warm]
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for i in range(args.steps):
        ctx.check(ctx.lib.cs_set_state(ctx.h, px, pv))
        ctx.step_async(p)
        ctx.check(ctx.lib.cs_get_state(ctx.h, px, pv))
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max_over_ranks(max(e0.elapsed_time(e1), wall * 1e3))
    e2e = {"value": node_steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": 2 * 12 * N,
           "d2h_bytes_per_step": 2 * 12 * N}

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_baseline(workload(args, 0, small=spec["single"]), args.cpu_seconds, "ref", 1)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms"] / args.steps, "higher_is_better": True,
            "scaling": "strong" if parts is not None else "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {
                "workload": args.workload if args.workload != "windy1024x64" else scene.name,
                "sheets": len(scene.sheets), "nodes_per_gpu": N, "nnzb_per_gpu": nnzb, "tol": args.tol,
                "scheme": "mixed FP32 PCG, FP64 dot products, FP64 residual replacements (reliable updates)",
                "warm_start": args.warm,
                "solver": args.solver,
                "precond": ("strip-local Chebyshev degree %d over block-Jacobi%s" %
                            (deg, " + coarse-space correction" if coarse else "")
                            if deg >= 3 and args.solver == "auto" else "block-Jacobi"),
                "l2": "inputs larger than L2 (system matrix %.2f GB per GPU)" % (sizes[3] * 36 / 1e9)
                      if sizes[3] * 36 > 126e6 else "system matrix %.3f GB per GPU: within L2" % (sizes[3] * 36 / 1e9),
                "parallelism": (f"one workload's sheets split over {world} ranks by stored blocks" if parts is not None
                                else f"sheets x{world} (no collective on the data path)"),
                "launch": "host loop" if args.host_loop else "CUDA graph with a device-driven while loop",
            },
            "iters_mean": best["iters_mean"], "iters_max": best["iters_max"],
            "converged_frac": best["converged_frac"], "max_relres": best["max_relres"],
            "arms": arms,
            "speedup_vs_plain_fp32": (value / plain["value"]) if plain else None,
            "plain_fp32_note": "plain FP32 PCG (block Jacobi, zero guess, batched loop streaming the system from "
                               "HBM) stops on its own FP32 recursive residual; converged_frac is the share of "
                               "sheets whose FP64-checked residual meets tol; dv_err_vs_fp64 is against an FP64 "
                               "direct solve of the arm's own assembled system on sampled sheets",
            "warm_start_training": train_info,
            "partition": part_info,
            "solver_plan": info,
            "tuning": tuning,
            "roofline": roofline,
            "roofline_smem": roof_smem,
            "roofline_batched_spmv": roof_spmv,
            "kernel_ms": prof,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": best["launches"],
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    ctx.close()
    group.close()


def run_detect(args):
    """Simulator::simulateStep's physics and collision parts on the device: proximity detection
    (Simulator.cu:571-586), the implicit step with the detected proximities (mixed precision,
    previous-step warm start) and the collision step (Simulator.cu:602-684), each call timed
    (detection and the collision step synchronise).  One JSON line."""
    import numpy as np
    sc = scenes_mod()
    from clothsimulator_b200 import native
    if args.detect == "windy":
        scene, groups = sc.windy_batch(args.sheets, args.nq, seed=eval_seed(0)), np.arange(args.sheets)
    elif args.detect in ("stacked", "crossing"):
        scene, groups = sc.stacked_sheets(256, n_layers=2, seed=1), None
        if args.detect == "crossing":
            scene.sheets[1]["v"] = scene.sheets[1]["v"].copy()
            scene.sheets[1]["v"][:, 2] = -0.5
    else:
        scene, groups = sc.folded_sheet(256, seed=1), None
    ctx = native.Context(0).load(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol, max_iters=20000,
                           precision=native.PREC_MIXED, warm_start=native.WARM_PREVIOUS,
                           precond_degree=args.precond_degree)
    det, both, col, full, counts, impacts = [], [], [], [], [], []
    thickness = float(np.float32(0.1) * np.float32(1e-3))  # Magic::collisionThickness default
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        counts.append(ctx.detect_proximities(1e-3, groups=groups))
        t1 = time.perf_counter()
        stats, _ = ctx.step(p, allow_unconverged=True)
        ctx.sync()
        t2 = time.perf_counter()
        rounds, imp, _ = ctx.collision_step(scene.dt, thickness, groups=groups, allow_unresolved=True)
        t3 = time.perf_counter()
        impacts.append(imp)
        if i >= args.warmup:
            det.append(1e3 * (t1 - t0))
            both.append(1e3 * (t2 - t0))
            col.append(1e3 * (t3 - t2))
            full.append(1e3 * (t3 - t0))
    out = {"mode": "detect", "workload": scene.name, "faces": scene.n_faces, "nodes": scene.n_nodes,
           "proximities": counts[-1], "steps": args.steps, "warmup": args.warmup,
           "detect_ms_median": float(np.median(det)), "detect_and_step_ms_median": float(np.median(both)),
           "collision_step_ms_median": float(np.median(col)), "impacts_last": impacts[-1],
           "detect_step_collide_ms_median": float(np.median(full)),
           "node_steps_per_s_with_contact": scene.n_nodes / (1e-3 * float(np.median(full))),
           "last_step_converged": int(stats.converged), "last_step_iters": int(stats.max_iters)}
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = parse()
    if args.detect:
        run_detect(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
