"""ctypes binding of libclothstep.so (the C ABI in include/clothstep.h).

This is plumbing for Python callers (tests, bench.py); it adds no computation.  The library
must be built in-tree (``python -c "import __graft_entry__; __graft_entry__.build()"`` or
``make -C clothsimulator_b200/csrc``); importing this module without it raises, and there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libclothstep.so")

CS_OK = 0
CS_ERR_INVALID_ARG = 1
CS_ERR_CUDA = 2
CS_ERR_NOT_CONVERGED = 3
CS_ERR_NON_SPD = 4
CS_ERR_TIMEOUT = 5
CS_ERR_STATE = 6
CS_ERR_NO_DEVICE = 7
CS_ERR_NOT_TRAINED = 8

PREC_PLAIN_FP32 = 0
PREC_MIXED = 1
WARM_ZERO, WARM_PREVIOUS, WARM_LEARNED, WARM_GIVEN = 0, 1, 2, 3
SOLVER_AUTO, SOLVER_BATCHED = 0, 1

EXPORTED = [
    "cs_create", "cs_destroy", "cs_last_error", "cs_load_batch", "cs_get_sizes", "cs_set_state", "cs_get_state",
    "cs_set_state_device", "cs_get_state_device", "cs_step", "cs_sync", "cs_set_warm_start", "cs_get_dv",
    "cs_get_instance_stats", "cs_assemble", "cs_get_system", "cs_get_element_forces", "cs_spmv",
    "cs_device_pointers", "cs_profile_kernels", "cs_get_counters", "cs_get_stream",
    "cs_solve_block_csr_noalloc", "cs_tc_gemm_check", "cs_mlp_init", "cs_mlp_record", "cs_mlp_fit_normalization",
    "cs_mlp_train", "cs_mlp_gradient", "cs_mlp_predict", "cs_mlp_get_record", "cs_mlp_get_weights",
    "cs_mlp_set_weights", "cs_get_solver_info", "cs_set_proximities", "cs_detect_proximities",
    "cs_get_proximities", "cs_collision_step", "cs_mlp_moments", "cs_mlp_set_moments", "cs_mlp_gradient_device",
    "cs_mlp_apply_gradient", "cs_get_resident_blocks", "cs_set_handle_motions", "cs_tune",
    "cs_mlp_train_step", "cs_mlp_energy_gradient", "cs_mlp_energy_begin", "cs_mlp_energy_gradient_device",
    "cs_mlp_energy_end", "cs_impact_order",
]
MLP_PARAMS = 14761
MLP_TRAINED = 14723


class MaterialDesc(ctypes.Structure):
    _fields_ = [
        ("density", ctypes.c_float),
        ("stretching", ctypes.c_float * 24),
        ("bending", ctypes.c_float * 15),
        ("thicken", ctypes.c_float),
        ("density_mult", ctypes.c_float),
        ("stretching_mult", ctypes.c_float),
        ("bending_mult", ctypes.c_float),
    ]


_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)
_dp = ctypes.POINTER(ctypes.c_double)


class SheetDesc(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int), ("n_verts", ctypes.c_int), ("n_faces", ctypes.c_int), ("n_handles", ctypes.c_int),
        ("x", _fp), ("v", _fp), ("uv", _fp), ("face_nodes", _ip), ("face_verts", _ip),
        ("handle_nodes", _ip), ("handle_pos", _fp), ("material", ctypes.c_int),
        ("wind_density", ctypes.c_float), ("wind_drag", ctypes.c_float), ("wind_velocity", ctypes.c_float * 3),
    ]


class StepParams(ctypes.Structure):
    _fields_ = [
        ("dt", ctypes.c_float), ("gravity", ctypes.c_float * 3), ("handle_stiffness", ctypes.c_float),
        ("tol", ctypes.c_double), ("inner_tol", ctypes.c_double), ("max_iters", ctypes.c_int),
        ("sweep_cap", ctypes.c_int), ("precision", ctypes.c_int), ("warm_start", ctypes.c_int),
        ("advance", ctypes.c_int), ("use_graph", ctypes.c_int), ("solver", ctypes.c_int),
        ("precond_degree", ctypes.c_int), ("coarse", ctypes.c_int),
        ("transformations", ctypes.POINTER(ctypes.c_float)), ("n_transformations", ctypes.c_int),
        ("warm_scale", ctypes.c_int),
    ]


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("spmv_ms", ctypes.c_float * 24), ("spmv_checksum", ctypes.c_uint32 * 24),
        ("spmv_threads", ctypes.c_int * 24), ("spmv_spw", ctypes.c_int * 24), ("spmv_unroll", ctypes.c_int * 24),
        ("precond_ms", ctypes.c_float * 6), ("precond_degree", ctypes.c_int * 6), ("precond_coarse", ctypes.c_int * 6),
        ("best_spmv", ctypes.c_int), ("best_precond", ctypes.c_int),
        ("solver_ms", ctypes.c_float * 2), ("best_solver", ctypes.c_int),
    ]


class StepStats(ctypes.Structure):
    _fields_ = [
        ("n_instances", ctypes.c_int), ("converged", ctypes.c_int), ("max_iters", ctypes.c_int),
        ("total_iters", ctypes.c_longlong), ("max_sweeps", ctypes.c_int), ("warm_rejected", ctypes.c_int),
        ("loop_trips", ctypes.c_int), ("max_rel_residual", ctypes.c_double), ("ms", ctypes.c_float),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# cs_proximity_desc, field for field (all 4-byte members: no padding)
PROXIMITY_DTYPE = np.dtype([
    ("nodes", "<i4", (4,)), ("x", "<f4", (4, 3)), ("v", "<f4", (4, 3)), ("mass", "<f4", (4,)),
    ("free_mask", "<i4"), ("normal", "<f4", (3,)), ("w", "<f4", (4,)), ("mu", "<f4"), ("stiffness", "<f4"),
])
assert PROXIMITY_DTYPE.itemsize == 168


def proximity_records(prox: dict) -> np.ndarray:
    """cs_proximity_desc array from a dict of arrays: nodes (n, 4) batch node ids or -1, x, v
    (n, 4, 3) and mass (n, 4) of the points outside the batch, free (n,) bit mask, normal
    (n, 3), w (n, 4), mu (n,), stiffness (n,)."""
    n = len(prox["mu"])
    rec = np.zeros(n, PROXIMITY_DTYPE)
    rec["nodes"] = np.asarray(prox["nodes"]).reshape(n, 4)
    rec["x"] = np.asarray(prox["x"]).reshape(n, 4, 3)
    rec["v"] = np.asarray(prox["v"]).reshape(n, 4, 3)
    rec["mass"] = np.asarray(prox["mass"]).reshape(n, 4)
    rec["free_mask"] = np.asarray(prox["free"]).reshape(n)
    rec["normal"] = np.asarray(prox["normal"]).reshape(n, 3)
    rec["w"] = np.asarray(prox["w"]).reshape(n, 4)
    rec["mu"] = np.asarray(prox["mu"]).reshape(n)
    rec["stiffness"] = np.asarray(prox["stiffness"]).reshape(n)
    return rec


class DetectParams(ctypes.Structure):
    _fields_ = [
        ("repulsion_thickness", ctypes.c_float), ("collision_stiffness", ctypes.c_float),
        ("friction", ctypes.c_float), ("sheet_group", ctypes.POINTER(ctypes.c_int32)),
    ]


class CollisionParams(ctypes.Structure):
    _fields_ = [("thickness", ctypes.c_float), ("dt", ctypes.c_float), ("sheet_group", ctypes.POINTER(ctypes.c_int32))]


class CollisionStats(ctypes.Structure):
    _fields_ = [("rounds", ctypes.c_int), ("impacts", ctypes.c_int)]


_LIB = None


def load_library() -> ctypes.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build()")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    sig = {
        "cs_create": [ctypes.POINTER(vp), ctypes.c_int],
        "cs_destroy": [vp],
        "cs_load_batch": [vp, ctypes.POINTER(MaterialDesc), ctypes.c_int, ctypes.POINTER(SheetDesc), ctypes.c_int],
        "cs_get_sizes": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "cs_get_solver_info": [vp, ctypes.POINTER(ctypes.c_int)],
        "cs_get_resident_blocks": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "cs_set_proximities": [vp, vp, ctypes.c_int, ctypes.c_float],
        "cs_detect_proximities": [vp, ctypes.POINTER(DetectParams), ctypes.POINTER(ctypes.c_int)],
        "cs_get_proximities": [vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)],
        "cs_collision_step": [vp, ctypes.POINTER(CollisionParams), ctypes.POINTER(CollisionStats)],
        "cs_set_state": [vp, _fp, _fp],
        "cs_set_handle_motions": [vp, _ip, ctypes.c_int],
        "cs_tune": [vp, ctypes.POINTER(StepParams), ctypes.c_int, vp],
        "cs_get_state": [vp, _fp, _fp],
        "cs_set_state_device": [vp, vp, vp],
        "cs_get_state_device": [vp, vp, vp],
        "cs_step": [vp, ctypes.POINTER(StepParams), ctypes.POINTER(StepStats)],
        "cs_sync": [vp],
        "cs_set_warm_start": [vp, _fp],
        "cs_get_dv": [vp, _fp],
        "cs_get_instance_stats": [vp, _ip, _dp, _ip],
        "cs_assemble": [vp, ctypes.POINTER(StepParams)],
        "cs_get_system": [vp, _ip, _ip, _fp, _fp],
        "cs_get_element_forces": [vp, _fp, _fp, _fp, _fp, _ip],
        "cs_spmv": [vp, _fp, _fp],
        "cs_device_pointers": [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)],
        "cs_profile_kernels": [vp, ctypes.POINTER(StepParams), ctypes.c_int, _fp],
        "cs_get_counters": [vp, ctypes.POINTER(ctypes.c_longlong)],
        "cs_get_stream": [vp, ctypes.POINTER(vp)],
        "cs_solve_block_csr_noalloc": [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int,
                                       vp, _ip, _dp],
        "cs_tc_gemm_check": [vp, vp, _fp, ctypes.c_int, ctypes.c_int],
        "cs_mlp_init": [vp, ctypes.c_int, ctypes.c_ulonglong],
        "cs_mlp_record": [vp, ctypes.c_int, ctypes.c_int],
        "cs_mlp_fit_normalization": [vp, ctypes.c_int],
        "cs_mlp_train": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int, ctypes.c_ulonglong, _fp],
        "cs_mlp_gradient": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _fp, _fp],
        "cs_mlp_train_step": [vp, ctypes.POINTER(StepParams), ctypes.c_float, ctypes.c_int, ctypes.c_ulonglong,
                              ctypes.POINTER(StepStats), _fp],
        "cs_mlp_energy_gradient": [vp, ctypes.POINTER(StepParams), ctypes.c_int, ctypes.c_int, _fp, _fp],
        "cs_mlp_energy_begin": [vp, ctypes.POINTER(StepParams)],
        "cs_mlp_energy_gradient_device": [vp, ctypes.c_int, ctypes.c_int, vp, _fp],
        "cs_mlp_energy_end": [vp, ctypes.POINTER(StepStats)],
        "cs_impact_order": [vp, _ip, _fp, _ip, ctypes.c_int, _ip],
        "cs_mlp_moments": [vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_longlong)],
        "cs_mlp_set_moments": [vp, _dp, ctypes.c_longlong],
        "cs_mlp_gradient_device": [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, _fp],
        "cs_mlp_apply_gradient": [vp, vp, ctypes.c_float],
        "cs_mlp_predict": [vp, _fp],
        "cs_mlp_get_record": [vp, ctypes.c_int, _fp, _fp],
        "cs_mlp_get_weights": [vp, _fp, ctypes.c_int],
        "cs_mlp_set_weights": [vp, _fp, ctypes.c_int],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.cs_last_error.argtypes = [vp]
    lib.cs_last_error.restype = ctypes.c_char_p
    _LIB = lib
    return lib


class ClothStepError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"status {status}: {message}")
        self.status = status


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def material_desc(spec: dict) -> MaterialDesc:
    m = MaterialDesc()
    m.density = spec["density"]
    st = np.asarray(spec["stretching"], np.float32).reshape(24)
    be = np.asarray(spec["bending"], np.float32).reshape(15)
    for i in range(24):
        m.stretching[i] = st[i]
    for i in range(15):
        m.bending[i] = be[i]
    m.thicken = spec.get("thicken", 1.0)
    m.density_mult = spec.get("density_mult", 1.0)
    m.stretching_mult = spec.get("stretching_mult", 1.0)
    m.bending_mult = spec.get("bending_mult", 1.0)
    return m


def step_params(dt, gravity=(0.0, -9.8, 0.0), handle_stiffness=1e3, tol=1e-6, inner_tol=1e-2, max_iters=2000,
                sweep_cap=0, precision=PREC_MIXED, warm_start=WARM_ZERO, advance=1, use_graph=1,
                solver=0, precond_degree=1, coarse=1, warm_scale=0) -> StepParams:
    p = StepParams()
    p.dt = dt
    for i in range(3):
        p.gravity[i] = gravity[i]
    p.handle_stiffness = handle_stiffness
    p.tol = tol
    p.inner_tol = inner_tol
    p.max_iters = max_iters
    p.sweep_cap = sweep_cap
    p.precision = precision
    p.warm_start = warm_start
    p.advance = advance
    p.use_graph = use_graph
    p.solver = solver
    p.precond_degree = precond_degree
    p.coarse = coarse
    p.transformations = None
    p.n_transformations = 0
    p.warm_scale = warm_scale
    return p


TRANSFORM_FLOATS = 8


def set_transformations(p: StepParams, transforms) -> StepParams:
    """The motions' transformations of one step into p: an (n, 8) array of scaling, translation
    (3), rotation quaternion (s, x, y, z).  The array is kept alive on p."""
    t = np.ascontiguousarray(np.asarray(transforms, np.float32).reshape(-1, TRANSFORM_FLOATS))
    p._transforms = t
    p.transformations = t.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    p.n_transformations = t.shape[0]
    return p


class Context:
    """Owns one cs_ctx.  `sheets` are dicts as produced by clothsimulator_b200.scenes."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        st = self.lib.cs_create(ctypes.byref(h), device)
        if st != CS_OK:
            raise ClothStepError(st, "cs_create failed (no usable sm_100 CUDA device)")
        self.h = h
        self.device = device
        self._keep = []
        self.n = 0

    def check(self, st: int, allow=(CS_OK,)):
        if st not in allow:
            raise ClothStepError(st, self.lib.cs_last_error(self.h).decode())
        return st

    def close(self):
        if getattr(self, "h", None):
            self.lib.cs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, sheets):
        mats = (MaterialDesc * len(sheets))()
        descs = (SheetDesc * len(sheets))()
        keep = []
        for i, s in enumerate(sheets):
            mats[i] = material_desc(s["material"])
            d = descs[i]
            x, v, uv = _f32(s["x"]), _f32(s["v"]), _f32(s["uv"])
            fx, fu = _i32(s["fx"]), _i32(s["fu"])
            hn = _i32(s.get("handles", np.zeros(0, np.int32)))
            keep += [x, v, uv, fx, fu, hn]
            d.n_nodes = x.shape[0]
            d.n_verts = uv.shape[0]
            d.n_faces = fx.shape[0]
            d.n_handles = hn.shape[0]
            d.x = x.ctypes.data_as(_fp)
            d.v = v.ctypes.data_as(_fp)
            d.uv = uv.ctypes.data_as(_fp)
            d.face_nodes = fx.ctypes.data_as(_ip)
            d.face_verts = fu.ctypes.data_as(_ip)
            d.handle_nodes = hn.ctypes.data_as(_ip)
            d.handle_pos = None
            d.material = i
            w = s["wind"]
            d.wind_density = w["density"]
            d.wind_drag = w["drag"]
            for k in range(3):
                d.wind_velocity[k] = w["velocity"][k]
        self.check(self.lib.cs_load_batch(self.h, mats, len(sheets), descs, len(sheets)))
        self.sizes = self.get_sizes()
        self.n = int(self.sizes[0])
        self.n_sheets = len(sheets)
        return self

    def get_sizes(self):
        s = (ctypes.c_longlong * 7)()
        self.check(self.lib.cs_get_sizes(self.h, s))
        return [int(v) for v in s]

    def solver_info(self) -> dict:
        """Cluster-resident solve plan of the loaded batch."""
        s = (ctypes.c_int * 11)()
        self.check(self.lib.cs_get_solver_info(self.h, s))
        keys = ("resident_sheets", "ctas_per_cluster", "threads_per_cta", "clusters", "panels_in_smem", "smem_bytes",
                "spmv_threads_per_block", "spmv_slices_per_warp", "spmv_slots_loaded_together",
                "tuned_precond_degree", "tuned_coarse")
        return dict(zip(keys, [int(v) for v in s]))

    def tune(self, params: StepParams, reps: int = 10) -> dict:
        """cs_tune: times the batched SpMV's launch shapes and the resident preconditioners on the
        loaded batch; the fastest SpMV shape is used from then on."""
        r = TuneResult()
        self.check(self.lib.cs_tune(self.h, ctypes.byref(params), reps, ctypes.byref(r)))
        shapes = [{"threads": r.spmv_threads[k], "slices_per_warp": r.spmv_spw[k], "unroll": r.spmv_unroll[k],
                   "ms": float(r.spmv_ms[k]), "checksum": int(r.spmv_checksum[k])} for k in range(24)]
        pre = [{"degree": r.precond_degree[k], "coarse": r.precond_coarse[k], "ms": float(r.precond_ms[k])}
               for k in range(6)]
        return {"spmv": shapes, "best_spmv": r.best_spmv, "precond": pre, "best_precond": r.best_precond,
                "solver_ms": {"auto": float(r.solver_ms[0]), "batched": float(r.solver_ms[1])},
                "best_solver": "auto" if r.best_solver == SOLVER_AUTO else "batched"}

    def resident_blocks(self) -> dict:
        """Blocks of the resident sheets' systems, the strip-local ones (read by each local SpMV
        of the Chebyshev preconditioner), and the power iterations per resident solve."""
        s = (ctypes.c_longlong * 3)()
        self.check(self.lib.cs_get_resident_blocks(self.h, s))
        return {"blocks": int(s[0]), "local_blocks": int(s[1]), "power_iters": int(s[2])}

    def set_proximities(self, prox: dict | None, thickness: float = 0.0):
        """Proximities of the following steps (None or an empty dict clears them); see
        proximity_records for the arrays."""
        rec = proximity_records(prox) if prox and len(prox["mu"]) else np.zeros(0, PROXIMITY_DTYPE)
        self._prox = rec  # kept alive for the call only; the library copies it
        self.check(self.lib.cs_set_proximities(self.h, rec.ctypes.data if len(rec) else None, len(rec),
                                               float(thickness)))
        self.sizes = self.get_sizes()

    def detect_proximities(self, repulsion_thickness: float = 1e-3, collision_stiffness: float = 1e9,
                           friction: float = 0.6, groups=None) -> int:
        """Detects proximities among the sheets' current states on the device and sets them
        (cs_detect_proximities); sheets with equal `groups` entries interact (all when None).
        Returns how many were found."""
        g = None if groups is None else np.ascontiguousarray(groups, np.int32)
        p = DetectParams(repulsion_thickness, collision_stiffness, friction,
                         g.ctypes.data_as(_ip) if g is not None else None)
        n = ctypes.c_int(0)
        self.check(self.lib.cs_detect_proximities(self.h, ctypes.byref(p), ctypes.byref(n)))
        self.sizes = self.get_sizes()
        return n.value

    def collision_step(self, dt: float, thickness: float = 1e-4, groups=None, allow_unresolved: bool = False):
        """The collision step after cs_step (cs_collision_step): impacts between the positions at
        the start of the last step and the current ones are resolved, then v = (x - x0) / dt.
        Returns (rounds, impacts, status)."""
        g = None if groups is None else np.ascontiguousarray(groups, np.int32)
        p = CollisionParams(thickness, dt, g.ctypes.data_as(_ip) if g is not None else None)
        s = CollisionStats()
        allow = (CS_OK, CS_ERR_NOT_CONVERGED) if allow_unresolved else (CS_OK,)
        st = self.check(self.lib.cs_collision_step(self.h, ctypes.byref(p), ctypes.byref(s)), allow)
        return s.rounds, s.impacts, st

    def get_proximities(self) -> dict:
        """The proximities in force, as a dict of arrays (see proximity_records)."""
        n = ctypes.c_int(0)
        self.check(self.lib.cs_get_proximities(self.h, None, 0, ctypes.byref(n)))
        rec = np.zeros(n.value, PROXIMITY_DTYPE)
        if n.value:
            self.check(self.lib.cs_get_proximities(self.h, rec.ctypes.data, n.value, ctypes.byref(n)))
        return {"nodes": rec["nodes"].copy(), "x": rec["x"].copy(), "v": rec["v"].copy(), "mass": rec["mass"].copy(),
                "free": rec["free_mask"].copy(), "normal": rec["normal"].copy(), "w": rec["w"].copy(),
                "mu": rec["mu"].copy(), "stiffness": rec["stiffness"].copy()}

    def set_handle_motions(self, motion):
        """The motion of every handle (-1: fixed), the sheets' handles in load order."""
        m = _i32(motion)
        self.check(self.lib.cs_set_handle_motions(self.h, m.ctypes.data_as(_ip), m.shape[0]))

    def set_state(self, x=None, v=None):
        xa = _f32(x) if x is not None else None
        va = _f32(v) if v is not None else None
        self.check(self.lib.cs_set_state(self.h, xa.ctypes.data_as(_fp) if xa is not None else None,
                                         va.ctypes.data_as(_fp) if va is not None else None))
        self.check(self.lib.cs_sync(self.h))

    def get_state(self):
        x = np.zeros((self.n, 3), np.float32)
        v = np.zeros((self.n, 3), np.float32)
        self.check(self.lib.cs_get_state(self.h, x.ctypes.data_as(_fp), v.ctypes.data_as(_fp)))
        return x, v

    def step(self, params: StepParams, allow_unconverged: bool = False):
        stats = StepStats()
        allow = (CS_OK, CS_ERR_NOT_CONVERGED, CS_ERR_NON_SPD) if allow_unconverged else (CS_OK,)
        st = self.check(self.lib.cs_step(self.h, ctypes.byref(params), ctypes.byref(stats)), allow)
        return stats, st

    def step_async(self, params: StepParams):
        self.check(self.lib.cs_step(self.h, ctypes.byref(params), None))

    def sync(self):
        self.check(self.lib.cs_sync(self.h))

    def set_warm_start(self, dv):
        a = _f32(dv)
        self.check(self.lib.cs_set_warm_start(self.h, a.ctypes.data_as(_fp)))

    def get_dv(self):
        dv = np.zeros((self.n, 3), np.float32)
        self.check(self.lib.cs_get_dv(self.h, dv.ctypes.data_as(_fp)))
        return dv

    def instance_stats(self):
        S = self.n_sheets
        it = np.zeros(S, np.int32)
        rr = np.zeros(S, np.float64)
        fl = np.zeros(S, np.int32)
        self.check(self.lib.cs_get_instance_stats(self.h, it.ctypes.data_as(_ip), rr.ctypes.data_as(_dp),
                                                  fl.ctypes.data_as(_ip)))
        return it, rr, fl

    def assemble(self, params: StepParams):
        self.check(self.lib.cs_assemble(self.h, ctypes.byref(params)))

    def system(self):
        nnzb = self.sizes[6]
        rp = np.zeros(self.n + 1, np.int32)
        ci = np.zeros(nnzb, np.int32)
        val = np.zeros((nnzb, 3, 3), np.float32)
        b = np.zeros(3 * self.n, np.float32)
        self.check(self.lib.cs_get_system(self.h, rp.ctypes.data_as(_ip), ci.ctypes.data_as(_ip),
                                          val.ctypes.data_as(_fp), b.ctypes.data_as(_fp)))
        return rp, ci, val, b

    def element_forces(self):
        F, E = self.sizes[1], self.sizes[2]
        ff = np.zeros((F, 9), np.float32)
        fJ = np.zeros((F, 9, 9), np.float32)
        ef = np.zeros((E, 12), np.float32)
        eJ = np.zeros((E, 12, 12), np.float32)
        en = np.zeros((E, 4), np.int32)
        self.check(self.lib.cs_get_element_forces(self.h, ff.ctypes.data_as(_fp), fJ.ctypes.data_as(_fp),
                                                  ef.ctypes.data_as(_fp), eJ.ctypes.data_as(_fp),
                                                  en.ctypes.data_as(_ip)))
        return ff, fJ, ef, eJ, en

    def spmv(self, x):
        xa = _f32(x).reshape(-1)
        y = np.zeros_like(xa)
        self.check(self.lib.cs_spmv(self.h, xa.ctypes.data_as(_fp), y.ctypes.data_as(_fp)))
        return y

    def device_pointers(self):
        x, v, dv = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        self.check(self.lib.cs_device_pointers(self.h, ctypes.byref(x), ctypes.byref(v), ctypes.byref(dv)))
        return x.value, v.value, dv.value

    # cs_profile_kernels' entries; the first (a separate face kernel) stays 0 since the assembly
    # gather evaluates the face terms itself, and is left out
    KERNELS = [None, "edge", "gather", "spmv", "vector", "reduce", "spmv_fp64", "resident_solve", "coarse_setup",
               "batched_coarse_setup", "batched_coarse_trip"]

    def profile_kernels(self, params: StepParams, reps: int = 20) -> dict:
        ms = (ctypes.c_float * 11)()
        self.check(self.lib.cs_profile_kernels(self.h, ctypes.byref(params), reps, ms))
        return {k: float(ms[i]) for i, k in enumerate(self.KERNELS) if k is not None}

    def counters(self):
        out = (ctypes.c_longlong * 3)()
        self.check(self.lib.cs_get_counters(self.h, out))
        return {"steps": int(out[0]), "trips": int(out[1]), "launches": int(out[2])}

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self.check(self.lib.cs_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    # --- learned warm start -------------------------------------------------------------
    def mlp_init(self, slots: int, seed: int = 0):
        self.check(self.lib.cs_mlp_init(self.h, slots, seed))

    def mlp_record(self, slot: int, what: int):
        self.check(self.lib.cs_mlp_record(self.h, slot, what))

    def mlp_fit_normalization(self, n_slots: int):
        self.check(self.lib.cs_mlp_fit_normalization(self.h, n_slots))

    def mlp_train(self, n_slots: int, epochs: int, lr: float = 1e-3, sheets_per_batch: int = 64, seed: int = 0):
        losses = np.zeros(epochs, np.float32)
        self.check(self.lib.cs_mlp_train(self.h, n_slots, epochs, lr, sheets_per_batch, seed,
                                         losses.ctypes.data_as(_fp)))
        return losses

    def mlp_gradient(self, slot: int, s0: int, s1: int):
        g = np.zeros(MLP_TRAINED, np.float32)
        loss = ctypes.c_float(0)
        self.check(self.lib.cs_mlp_gradient(self.h, slot, s0, s1, g.ctypes.data_as(_fp), ctypes.byref(loss)))
        return g, loss.value

    @property
    def torch_device(self):
        import torch

        return torch.device("cuda", self.device)

    def mlp_moments(self, n_slots: int):
        """Normalisation moment sums (38) and node count of the recorded slots."""
        sums = np.zeros(38, np.float64)
        n = ctypes.c_longlong(0)
        self.check(self.lib.cs_mlp_moments(self.h, n_slots, sums.ctypes.data_as(_dp), ctypes.byref(n)))
        return sums, n.value

    def mlp_set_moments(self, sums, count: int):
        a = np.ascontiguousarray(sums, np.float64)
        self.check(self.lib.cs_mlp_set_moments(self.h, a.ctypes.data_as(_dp), int(count)))

    def mlp_train_step(self, params: StepParams, lr: float = 1e-3, sheets_per_batch: int = 64, seed: int = 0,
                       allow_unconverged: bool = False):
        """cs_mlp_train_step: one step of the batch with energy-norm Adam updates between the
        solve and the state update.  Returns (stats, mean minibatch loss)."""
        stats = StepStats()
        loss = ctypes.c_float(0.0)
        st = self.lib.cs_mlp_train_step(self.h, ctypes.byref(params), lr, sheets_per_batch, seed, ctypes.byref(stats),
                                        ctypes.byref(loss))
        self.check(st, (CS_OK, CS_ERR_NOT_CONVERGED, CS_ERR_NON_SPD) if allow_unconverged else (CS_OK,))
        return stats, loss.value

    def mlp_energy_gradient(self, params: StepParams, s0: int, s1: int):
        """cs_mlp_energy_gradient: the energy-norm loss's gradient and value for sheets [s0, s1)."""
        g = np.zeros(MLP_TRAINED, np.float32)
        loss = ctypes.c_float(0)
        self.check(self.lib.cs_mlp_energy_gradient(self.h, ctypes.byref(params), s0, s1, g.ctypes.data_as(_fp),
                                                   ctypes.byref(loss)))
        return g, loss.value

    def impact_order(self, nodes, t, types):
        """cs_impact_order: the collision step's order of the given impacts (indices)."""
        nd = _i32(np.asarray(nodes).reshape(-1, 4))
        tt = _f32(t)
        ty = _i32(types)
        n = tt.shape[0]
        out = np.zeros(n, np.int32)
        self.check(self.lib.cs_impact_order(self.h, nd.ctypes.data_as(_ip), tt.ctypes.data_as(_fp),
                                            ty.ctypes.data_as(_ip), n, out.ctypes.data_as(_ip)))
        return out

    def mlp_energy_begin(self, params: StepParams):
        self.check(self.lib.cs_mlp_energy_begin(self.h, ctypes.byref(params)))

    def mlp_energy_gradient_device(self, s0: int, s1: int, grad) -> float:
        """The energy loss's gradient for sheets [s0, s1) into `grad` (a CUDA tensor of
        MLP_TRAINED floats on this context's device); returns the minibatch loss."""
        loss = ctypes.c_float(0.0)
        self.check(self.lib.cs_mlp_energy_gradient_device(self.h, s0, s1, ctypes.c_void_p(grad.data_ptr()),
                                                          ctypes.byref(loss)))
        return loss.value

    def mlp_energy_end(self, allow_unconverged: bool = False):
        stats = StepStats()
        st = self.lib.cs_mlp_energy_end(self.h, ctypes.byref(stats))
        self.check(st, (CS_OK, CS_ERR_NOT_CONVERGED, CS_ERR_NON_SPD) if allow_unconverged else (CS_OK,))
        return stats

    def mlp_gradient_device(self, slot: int, s0: int, s1: int, grad) -> float:
        """One minibatch's gradient into `grad`, a CUDA tensor of MLP_TRAINED floats on this
        context's device; returns the minibatch loss."""
        loss = ctypes.c_float(0.0)
        self.check(self.lib.cs_mlp_gradient_device(self.h, slot, s0, s1, ctypes.c_void_p(grad.data_ptr()),
                                                   ctypes.byref(loss)))
        return loss.value

    def mlp_apply_gradient(self, grad, lr: float):
        """The Adam step of cs_mlp_train with the gradient in `grad` (CUDA tensor)."""
        self.check(self.lib.cs_mlp_apply_gradient(self.h, ctypes.c_void_p(grad.data_ptr()), lr))

    def mlp_predict(self):
        p = np.zeros((self.n, 3), np.float32)
        self.check(self.lib.cs_mlp_predict(self.h, p.ctypes.data_as(_fp)))
        return p

    def mlp_get_record(self, slot: int):
        f = np.zeros((self.n, 16), np.float32)
        t = np.zeros((self.n, 3), np.float32)
        self.check(self.lib.cs_mlp_get_record(self.h, slot, f.ctypes.data_as(_fp), t.ctypes.data_as(_fp)))
        return f, t

    def mlp_get_weights(self):
        w = np.zeros(MLP_PARAMS, np.float32)
        self.check(self.lib.cs_mlp_get_weights(self.h, w.ctypes.data_as(_fp), MLP_PARAMS))
        return w

    def mlp_set_weights(self, w):
        a = _f32(w)
        self.check(self.lib.cs_mlp_set_weights(self.h, a.ctypes.data_as(_fp), MLP_PARAMS))
