"""Benchmark of the implicit cloth step on B200.

Workload (default): 1,024 sheets of 64x64 quads (4,326,400 nodes), top edge pinned, per-sheet
horizontal wind, stretching log-U[10, 500] N/m and bending log-U[1e-6, 1e-3] N m through the
material multipliers, dt = 1/100 s: the learned-warm-start configuration, which fits one GPU.
One step = assembly + batched PCG to an FP64-checked relative residual of 1e-6 for every sheet
+ v += dv, x += dt v, with the state resident in HBM.

Metric: node-steps/s (sum over sheets of nodes x steps / device time).  The line reports the
mixed-precision solver with its warm start (`value`: cluster-resident solve, strip-local
Chebyshev preconditioner of degree `--precond-degree`, reliable updates) and, in `arms`, the
same solver from other starts and with block-Jacobi, and plain FP32 PCG from a zero guess on
the same GPU.  `--impl reference` times the reference's CPU path for this
workload (the reference's own force code compiled from its sources + FP32 sparse Cholesky).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       torchrun --nproc-per-node N bench.py --gpus N   (one rank per GPU, sheets per rank fixed)
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sheets", type=int, default=1024)
    ap.add_argument("--nq", type=int, default=64)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--warm", default="learned", choices=["previous", "zero", "learned"])
    ap.add_argument("--solver", default="auto", choices=["auto", "batched"],
                    help="auto: sheets that fit a cluster's shared memory are solved cluster-resident")
    ap.add_argument("--precond-degree", type=int, default=3,
                    help="cluster-resident solver's preconditioner: 1 block-Jacobi, odd 3..15 a strip-local "
                         "Chebyshev polynomial of that degree (the batched loop always uses block-Jacobi)")
    ap.add_argument("--train-sheets", type=int, default=256, help="sheets of the training trajectories")
    ap.add_argument("--train-steps", type=int, default=24, help="recorded steps per training trajectory")
    ap.add_argument("--epochs", type=int, default=16)
    ap.add_argument("--weights", default="", help="load trained warm-start weights instead of training")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 arm")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--detect", default="", choices=["", "windy", "stacked", "folded", "crossing"],
                    help="time proximity detection, the step and the collision step on a contact workload "
                         "instead: windy = the 1,024-sheet batch, a group per sheet; stacked = two 256x256 "
                         "sheets 1.5 mm apart; folded = one 256x256 sheet folded onto itself; crossing = "
                         "stacked with the upper sheet moving down at 0.5 m/s")
    ap.add_argument("--host-loop", action="store_true",
                    help="launch the solve loop from the host instead of the CUDA graph (profilers cannot "
                         "see kernels inside a graph with conditional nodes)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class RankGroup:
    """One process per GPU (torchrun).  Sheets are independent, so ranks exchange no data:
    the group carries only the barriers around the timed region and the max over ranks of
    the device times (gloo, host scalars)."""

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

    def device_allreduce(self):
        """An in-place sum of CUDA tensors over the ranks: NCCL over NVLink (a group of its own
        beside the gloo group of the host scalars)."""
        if not self.dist:
            return None
        if getattr(self, "_nccl", None) is None:
            self._nccl = self.dist.new_group(backend="nccl")
        grp = self._nccl
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


def workload(args, rank):
    return scenes_mod().windy_batch(args.sheets, args.nq, seed=eval_seed(rank))


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
    scene = workload(args, 0)
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(1, args.warmup)):
        cpu_baseline(scene, 2.0, "ref", threads)
    samples = []
    for _ in range(args.steps):
        r = cpu_baseline(scene, args.cpu_seconds / max(1, args.steps) * 4, "ref", threads)
        vals.append(r["value"])
        samples.append(r["sample"])
    value = statistics.median(vals)
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": scene.name, "sheets": len(scene.sheets), "nodes": scene.n_nodes, "tol": args.tol},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": r["kind"], "sample": samples[-1]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch

    from clothsimulator_b200 import native

    group = RankGroup()
    rank, world, local = group.rank, group.world, group.local
    torch.cuda.set_device(local)
    scene = workload(args, rank)
    ctx = native.Context(local)
    ctx.load(scene.sheets)
    sizes = ctx.sizes
    N = sizes[0]
    x0 = np.concatenate([s["x"] for s in scene.sheets])
    v0 = np.concatenate([s["v"] for s in scene.sheets])
    stream = torch.cuda.ExternalStream(ctx.stream(), device=torch.device("cuda", local))

    barrier = group.barrier
    max_over_ranks = group.max

    # Learned warm start: trained on the device on separate seeded trajectories (the
    # evaluated workload's seeds are held out), or loaded from --weights.
    train_info = None
    if args.warm == "learned":
        t0 = time.perf_counter()
        if args.weights:
            weights = np.fromfile(args.weights, dtype=np.float32)
            train_info = {"source": args.weights}
        else:
            tscene = scenes_mod().windy_batch(args.train_sheets, args.nq, seed=train_seed(rank))
            tctx = native.Context(local)
            tctx.load(tscene.sheets)
            tctx.mlp_init(args.train_steps, 1)  # the same initial weights on every rank
            tp = native.step_params(tscene.dt, tscene.gravity, tscene.handle_stiffness, tol=1e-7, max_iters=8000)
            for _ in range(2):
                tctx.step(tp, allow_unconverged=True)
                tp.warm_start = native.WARM_PREVIOUS
            for t in range(args.train_steps):
                tctx.assemble(tp)
                tctx.mlp_record(t, 0)
                tctx.step(tp, allow_unconverged=True)
                tctx.mlp_record(t, 1)
            if world == 1:
                tctx.mlp_fit_normalization(args.train_steps)
                losses = tctx.mlp_train(args.train_steps, args.epochs, lr=1e-3, sheets_per_batch=32, seed=3)
            else:
                # data parallel: every rank trains on its own trajectories, gradients summed over
                # NCCL and averaged, normalisation from the moments summed over the ranks
                from clothsimulator_b200 import training

                losses = training.train_data_parallel(tctx, args.train_steps, args.train_sheets, args.epochs, 1e-3,
                                                      32, 3, allreduce_sum=group.device_allreduce(), world=world,
                                                      sum_host=group.sum_host)
            weights = tctx.mlp_get_weights()
            tctx.close()
            train_info = {"sheets": args.train_sheets, "steps": args.train_steps, "epochs": args.epochs,
                          "seeds": "disjoint from the evaluated workload",
                          "loss_first": float(losses[0]), "loss_last": float(losses[-1])}
            if world > 1:
                digest = float(np.float64(weights).sum())
                train_info["data_parallel"] = {
                    "ranks": world, "gradients": "NCCL all-reduce, averaged",
                    "weights_identical": group.max(digest) == -group.max(-digest)}
        train_info["seconds"] = time.perf_counter() - t0
        ctx.mlp_init(0, 0)
        ctx.mlp_set_weights(weights)

    solver_code = {"auto": native.SOLVER_AUTO, "batched": native.SOLVER_BATCHED}

    def timed_arm(precision, warm, solver, clocks=None, degree=args.precond_degree):
        ctx.set_state(x0, v0)
        p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol, max_iters=4000,
                               precision=precision, warm_start=native.WARM_ZERO, use_graph=0 if args.host_loop else 1,
                               solver=solver_code[solver], precond_degree=degree)
        for i in range(args.warmup):
            ctx.step(p, allow_unconverged=True)
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
        # one untimed step with statistics for the report
        ctx.step(p, allow_unconverged=True)
        it, rr, fl = ctx.instance_stats()
        return {
            "value": aggregate_value(N, args.steps, world, ms),
            "ms": ms,
            "ms_per_step": ms / args.steps,
            "launches": c1["launches"] - c0["launches"],
            "iters_mean": float(it.mean()),
            "iters_max": int(it.max()),
            "converged_frac": float(np.mean((fl & 1) > 0)),
            "warm_rejected_frac": float(np.mean((fl & 2) > 0)),
            "max_relres": float(rr.max()),
        }

    keys = ("value", "ms_per_step", "iters_mean", "iters_max", "converged_frac", "warm_rejected_frac", "max_relres")
    warm_mode = {"previous": native.WARM_PREVIOUS, "zero": native.WARM_ZERO, "learned": native.WARM_LEARNED}[args.warm]
    clocks = {}
    best = timed_arm(native.PREC_MIXED, warm_mode, args.solver, clocks)
    node_steps = N * args.steps * world
    value = best["value"]
    head = f"mixed_{args.warm}_{args.solver}"
    arms = {head: dict({k: best[k] for k in keys}, precond_degree=args.precond_degree if args.solver == "auto" else 1)}
    if not args.no_plain:
        # the plain FP32 arms keep block-Jacobi (the reference's solver structure); the mixed arms
        # use --precond-degree, with block-Jacobi beside them
        deg = args.precond_degree
        for name, prec, warm, solver, d in [
                ("mixed_zero_auto", native.PREC_MIXED, native.WARM_ZERO, "auto", deg),
                ("mixed_previous_auto", native.PREC_MIXED, native.WARM_PREVIOUS, "auto", deg),
                ("mixed_learned_auto_block_jacobi", native.PREC_MIXED, native.WARM_LEARNED, "auto", 1),
                ("mixed_zero_auto_block_jacobi", native.PREC_MIXED, native.WARM_ZERO, "auto", 1),
                ("plain_fp32_zero_auto", native.PREC_PLAIN_FP32, native.WARM_ZERO, "auto", 1),
                ("mixed_previous_batched", native.PREC_MIXED, native.WARM_PREVIOUS, "batched", 1),
                ("plain_fp32_zero_batched", native.PREC_PLAIN_FP32, native.WARM_ZERO, "batched", 1)]:
            if name in arms or (warm == native.WARM_LEARNED and args.warm != "learned") or (d == deg and name.endswith("block_jacobi")):
                continue
            r = timed_arm(prec, warm, solver, degree=d)
            arms[name] = dict({k: r[k] for k in keys}, precond_degree=d if solver == "auto" else 1)
    plain = arms.get("plain_fp32_zero_batched")

    # Rooflines, timed live on the context's stream (cs_profile_kernels).  The dominant kernel
    # of the default (resident) solver is cs_resident_pcg_kernel: its algorithmic bytes per
    # launch are the CG iterations it ran times the bytes one SpMV iteration moves (stored
    # blocks x 40 B + nodes x 48 B, the same per-iteration figure as the batched SpMV's), plus
    # the Chebyshev preconditioner's strip-local SpMVs at the same rate over the strip-local
    # blocks; the resident kernel serves them from shared memory, so its DRAM traffic is far
    # below them.
    prof = ctx.profile_kernels(native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol,
                                                  max_iters=4000, precond_degree=args.precond_degree), reps=5)
    it_res, _, _ = ctx.instance_stats()
    nnzb = sizes[6]
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0

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
                 "kernel": "cs_spmv_kernel", "bytes_per_launch": spmv_bytes, "ms_per_launch": prof["spmv"]}
    roof_res = None
    if prof["resident_solve"] > 0:
        per_sheet = np.array([(s_["fx"].shape[0], s_["x"].shape[0]) for s_ in scene.sheets], np.float64)
        nnzb_sheet = nnzb / len(scene.sheets)  # identical topologies in this workload
        # a CG iteration is one full SpMV plus, with the strip-local Chebyshev preconditioner,
        # (degree - 1) SpMVs over the strip-local blocks; each solve adds the power iterations
        rb = ctx.resident_blocks()
        local_frac = rb["local_blocks"] / max(rb["blocks"], 1)
        local_spmvs = it_res * (args.precond_degree - 1) + rb["power_iters"] if args.precond_degree >= 3 else 0 * it_res
        res_bytes = float(np.sum(it_res * (nnzb_sheet * 40 + per_sheet[:, 1] * 48)
                                 + local_spmvs * (local_frac * nnzb_sheet * 40 + per_sheet[:, 1] * 48)))
        res_achieved = res_bytes / (prof["resident_solve"] * 1e-3) / 1e9
        roof_res = {"bound": "hbm", "achieved": res_achieved, "peak": peak, "unit": "GB/s",
                    "frac": res_achieved / peak,
                    "traffic": traffic_per_launch("cs_resident_pcg_kernel_windy32x64_traffic.json", len(scene.sheets)),
                    "kernel": "cs_resident_pcg_kernel", "bytes_per_launch": res_bytes,
                    "ms_per_launch": prof["resident_solve"], "cg_iterations_per_launch": int(it_res.sum()),
                    "local_spmvs_per_launch": int(np.sum(local_spmvs)), "local_block_frac": local_frac,
                    "note": "per-iteration operands served from shared memory: achieved is the rate at which the "
                            "solve consumes SpMV bytes (the CG SpMVs and the Chebyshev preconditioner's strip-local "
                            "SpMVs), against the HBM roofline of the streaming formulation; above 1 means faster than "
                            "any solve that streams the system from HBM could run"}
    roofline = roof_res if (roof_res and args.solver == "auto") else roof_spmv

    # end to end through the C ABI with pinned host buffers: H2D of x, v, step, D2H of x, v
    hx = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
    hv = torch.empty((N, 3), dtype=torch.float32, pin_memory=True)
    hx.numpy()[:] = x0
    hv.numpy()[:] = v0
    fp = native._fp
    import ctypes as C

    px = C.cast(hx.data_ptr(), fp)
    pv = C.cast(hv.data_ptr(), fp)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=args.tol, max_iters=4000,
                           precision=native.PREC_MIXED, warm_start=native.WARM_ZERO, use_graph=0 if args.host_loop else 1,
                           solver=solver_code[args.solver], precond_degree=args.precond_degree)
    ctx.set_state(x0, v0)
    for i in range(args.warmup):
        ctx.check(ctx.lib.cs_set_state(ctx.h, px, pv))
        ctx.step(p, allow_unconverged=True)
        ctx.check(ctx.lib.cs_get_state(ctx.h, px, pv))
        p.warm_start = warm_mode
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
        cpu = cpu_baseline(scene, args.cpu_seconds, "ref", 1)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {
                "workload": scene.name, "sheets": len(scene.sheets), "nq": args.nq, "nodes_per_gpu": N,
                "nnzb_per_gpu": nnzb, "tol": args.tol,
                "scheme": "mixed FP32 PCG, FP64 dot products, FP64 residual replacements (reliable updates)",
                "warm_start": args.warm,
                "solver": args.solver,
                "precond": ("strip-local Chebyshev degree %d over block-Jacobi" % args.precond_degree
                            if args.precond_degree >= 3 and args.solver == "auto" else "block-Jacobi"),
                "l2": "inputs larger than L2 (system matrix %.2f GB per GPU)" % (sizes[3] * 36 / 1e9),
                "parallelism": f"sheets x{world} (no collective on the data path)",
                "launch": "host loop" if args.host_loop else "CUDA graph with a device-driven while loop",
            },
            "iters_mean": best["iters_mean"], "iters_max": best["iters_max"],
            "converged_frac": best["converged_frac"], "max_relres": best["max_relres"],
            "arms": arms,
            "speedup_vs_plain_fp32": (value / plain["value"]) if plain else None,
            "plain_fp32_note": "plain FP32 PCG (block Jacobi, zero guess, batched loop streaming the system from "
                               "HBM) stops on its own FP32 recursive residual; converged_frac is the share of "
                               "sheets whose FP64-checked residual meets tol",
            "warm_start_training": train_info,
            "solver_plan": ctx.solver_info(),
            "roofline": dict(roofline, peak_source="measured" if peaks else "fallback"),
            "roofline_batched_spmv": dict(roof_spmv, peak_source="measured" if peaks else "fallback"),
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
