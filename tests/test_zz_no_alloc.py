"""The allocation-free solve (cs_solve_block_csr_noalloc) against the batched solver.

Some callers cannot allocate device memory: hosts whose own allocator owns all device memory,
real-time loops that must not allocate, plugins that may not grow the device footprint.  For
them the library solves one block-CSR system with scratch in a fixed static device array.
This file runs last (pytest collects it last by name) so a failure here stops a `-x` run only
after every other test has run.  It must pass alone in a fresh process too.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from clothsimulator_b200 import native, scenes

TOL = 1e-6  # the parity tolerance used for solver outputs in the other GPU tests


def rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1)
    b = np.asarray(b, np.float64).reshape(-1)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _system(nq=40, seed=21):
    scene = scenes.hang(nq, seed=seed)
    s = scene.sheets[0]
    rng = np.random.default_rng(seed)
    s["x"] = (s["x"] + rng.normal(0, 0.01, s["x"].shape)).astype(np.float32)
    s["v"] = rng.normal(0, 0.1, s["v"].shape).astype(np.float32)
    ctx = native.Context(0)
    ctx.load(scene.sheets)
    p = native.step_params(scene.dt, scene.gravity, scene.handle_stiffness, tol=1e-10, max_iters=20000, advance=0)
    stats, _ = ctx.step(p)
    assert stats.converged == 1
    dv_ref = ctx.get_dv()
    rp, ci, val, b = ctx.system()
    return ctx, dv_ref, rp, ci, val, b


def _call(lib, n, nnzb, d_rp, d_ci, d_val, d_b, d_x, tol=1e-10, max_iters=20000, sync=True):
    it = ctypes.c_int(-1)
    rr = ctypes.c_double(-1.0)
    st = lib.cs_solve_block_csr_noalloc(n, nnzb, d_rp, d_ci, d_val, d_b, d_x, tol, max_iters, None,
                                        ctypes.byref(it) if sync else None, ctypes.byref(rr) if sync else None)
    return st, it.value, rr.value


def test_noalloc_solve_matches_batched_solver_twice():
    import torch

    ctx, dv_ref, rp, ci, val, b = _system()
    lib = native.load_library()
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rp).to(dev)
    d_ci = torch.from_numpy(ci).to(dev)
    d_val = torch.from_numpy(val.reshape(-1)).to(dev)
    d_b = torch.from_numpy(b).to(dev)
    n, nnzb = ctx.n, len(ci)
    for call in range(2):  # the second call reuses the scratch left by the first
        d_x = torch.full((3 * n,), float("nan"), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        st, it, rr = _call(lib, n, nnzb, d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                           d_x.data_ptr())
        assert st == native.CS_OK, f"call {call}: status {st}"
        assert it > 0 and 0 <= rr <= 1e-10
        x = d_x.cpu().numpy()
        assert rel(x, dv_ref) < TOL, f"call {call}"
    ctx.close()


def test_noalloc_rejects_oversized_and_malformed_input():
    import torch

    lib = native.load_library()
    dev = torch.device("cuda", 0)
    d = torch.zeros(64, dtype=torch.int32, device=dev)
    f = torch.zeros(64, dtype=torch.float32, device=dev)
    st, _, _ = _call(lib, 16385, 1, d.data_ptr(), d.data_ptr(), f.data_ptr(), f.data_ptr(), f.data_ptr())
    assert st == native.CS_ERR_INVALID_ARG
    # one row whose only column index points past the matrix: refused on the device before use
    rp = torch.tensor([0, 1], dtype=torch.int32, device=dev)
    ci = torch.tensor([5], dtype=torch.int32, device=dev)
    val = torch.eye(3, dtype=torch.float32, device=dev).reshape(-1)
    bb = torch.ones(3, dtype=torch.float32, device=dev)
    xx = torch.zeros(3, dtype=torch.float32, device=dev)
    st, _, _ = _call(lib, 1, 1, rp.data_ptr(), ci.data_ptr(), val.data_ptr(), bb.data_ptr(), xx.data_ptr())
    assert st == native.CS_ERR_INVALID_ARG


def test_noalloc_matches_fp64_oracle_and_reports_its_cap():
    """Against the FP64 direct solve of the same system (the CPU oracle), and with a cap of one
    iteration: CS_ERR_NOT_CONVERGED with one iteration reported."""
    import torch
    import pyoracle

    scene = scenes.hang(24, seed=5)
    s = scene.sheets[0]
    rng = np.random.default_rng(5)
    s["x"] = (s["x"] + rng.normal(0, 0.01, s["x"].shape)).astype(np.float32)
    s["v"] = rng.normal(0, 0.1, s["v"].shape).astype(np.float32)
    oc = pyoracle.Cloth(s, pyoracle.Material(s["material"], "float"))
    rp, ci, val, b = oc.assemble(scenes.step_params(scene, s))
    exact, _ = oc.solve(pyoracle.METHOD_LLT64)
    lib = native.load_library()
    dev = torch.device("cuda", 0)
    d_rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
    d_ci = torch.from_numpy(ci.astype(np.int32)).to(dev)
    d_val = torch.from_numpy(val.astype(np.float32).reshape(-1)).to(dev)
    d_b = torch.from_numpy(b.astype(np.float32)).to(dev)
    n = len(rp) - 1
    d_x = torch.zeros(3 * n, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    st, it, rr = _call(lib, n, len(ci), d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                       d_x.data_ptr())
    assert st == native.CS_OK and rr <= 1e-10
    assert rel(d_x.cpu().numpy(), exact) < TOL
    st, it, rr = _call(lib, n, len(ci), d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(), d_b.data_ptr(),
                       d_x.data_ptr(), max_iters=1)
    assert st == native.CS_ERR_NOT_CONVERGED and it == 1 and rr > 1e-10


def test_noalloc_asynchronous_form_on_a_stream():
    """The asynchronous form (no statistics pointers) on a non-default stream: it returns after
    the launch; after the stream is synchronised x holds the solution.  A system the device
    rejects leaves NaN in x."""
    import torch

    ctx, dv_ref, rp, ci, val, b = _system(nq=20, seed=9)
    lib = native.load_library()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        d_rp = torch.from_numpy(rp).to(dev)
        d_ci = torch.from_numpy(ci).to(dev)
        d_val = torch.from_numpy(val.reshape(-1)).to(dev)
        d_b = torch.from_numpy(b).to(dev)
        d_x = torch.zeros(3 * ctx.n, dtype=torch.float32, device=dev)
    st = lib.cs_solve_block_csr_noalloc(ctx.n, len(ci), d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(),
                                        d_b.data_ptr(), d_x.data_ptr(), 1e-10, 20000,
                                        ctypes.c_void_p(stream.cuda_stream), None, None)
    assert st == native.CS_OK
    stream.synchronize()
    assert rel(d_x.cpu().numpy(), dv_ref) < TOL
    # out-of-range column: the asynchronous form cannot report it, x becomes NaN
    with torch.cuda.stream(stream):
        bad_ci = d_ci.clone()
        bad_ci[0] = 10 * ctx.n
    st = lib.cs_solve_block_csr_noalloc(ctx.n, len(ci), d_rp.data_ptr(), bad_ci.data_ptr(), d_val.data_ptr(),
                                        d_b.data_ptr(), d_x.data_ptr(), 1e-10, 20000,
                                        ctypes.c_void_p(stream.cuda_stream), None, None)
    assert st == native.CS_OK
    stream.synchronize()
    assert np.all(np.isnan(d_x.cpu().numpy()))
    ctx.close()
