"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg, where
it is the checker, never the thing measured on the GPU path.  Two libraries share one
API shape:

* ``liboracle.so`` (prefix ``orc_``): the project's restatement of the reference's
  arithmetic (oracle_math.hpp, oracle_system.hpp), in float (the reference's FP32
  semantics) or double (the FP64 oracle);
* ``_ref/libclothref.so`` (prefix ``ref_``): the reference's own force, Jacobian,
  material and face code (PhysicsHelper.cu, Material.cu, Face.cu, Edge.cu, ...)
  compiled from its sources, with the oracle's assembly and solver around it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libclothref.so")
# The reference checkout's src/ directory, from which the adapter library is compiled: given by
# the CLOTHSIM_REFERENCE_SRC environment variable (the build entry point sets it where the
# checkout exists).  Only needed to build _ref/libclothref.so or to make the golden fixtures.
REFERENCE_ENV = "CLOTHSIM_REFERENCE_SRC"


def reference_src(required: bool = True) -> str | None:
    """The reference's src/ directory named by CLOTHSIM_REFERENCE_SRC.  Raises a clear error
    when it is required and unset or missing; returns None otherwise."""
    p = os.environ.get(REFERENCE_ENV, "")
    if p and os.path.isdir(p):
        return p
    if required:
        raise RuntimeError(f"{REFERENCE_ENV} must name the reference checkout's src/ directory "
                           f"(got {p!r})")
    return None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p

METHOD_LLT = 0      # LL^T in the cloth's precision: the reference CPU path
METHOD_LLT64 = 1    # LL^T in double of the same assembled system
METHOD_PCG64 = 2    # FP64 block-Jacobi PCG to a relative residual


def build(ref: bool = True) -> None:
    """Builds liboracle.so and, when the reference checkout is present, _ref/libclothref.so."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    src = reference_src(required=False) if ref else None
    if src:
        subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REFSRC={src}"], check=True)


def _d(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a, t):
    return a.ctypes.data_as(t)


class Lib:
    def __init__(self, which: str = "oracle"):
        self.which = which
        path = LIB_ORACLE if which == "oracle" else LIB_REF
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run oracle/pyoracle.build())")
        self.lib = ctypes.CDLL(path)
        self.p = "orc_" if which == "oracle" else "ref_"
        L = self.lib
        f = self.fn
        f("material_free", None, [_vp])
        f("material_density", ctypes.c_double, [_vp])
        f("material_stretching", None, [_vp, ctypes.c_int, _dp, _dp])
        f("material_bending", None, [_vp, ctypes.c_int, _dp, _dp])
        f("cloth_new", _vp, [_vp, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip])
        f("cloth_free", None, [_vp])
        f("cloth_num_edges", ctypes.c_int, [_vp])
        f("cloth_num_nodes", ctypes.c_int, [_vp])
        f("cloth_num_interior_edges", ctypes.c_int, [_vp])
        f("cloth_interior_edges", None, [_vp, _ip, _ip])
        f("cloth_face_forces", None, [_vp, _dp, _dp])
        f("cloth_edge_forces", None, [_vp, _dp, _dp, _dp])
        f("cloth_set_handles", None, [_vp, ctypes.c_int, _ip, _dp])
        f("cloth_assemble", ctypes.c_int, [_vp, _dp])
        f("cloth_system", None, [_vp, _ip, _ip, _dp, _dp])
        f("cloth_solve", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp])
        f("cloth_advance", None, [_vp, _dp, ctypes.c_double])
        f("cloth_state", None, [_vp, _dp, _dp])
        f("cloth_set_state", None, [_vp, _dp, _dp])
        f("cloth_masses", None, [_vp, _dp])
        f("cloth_normals", None, [_vp, _dp])
        f("cloth_step", ctypes.c_int, [_vp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp])
        f("cloth_factor_nnz", ctypes.c_longlong, [_vp])
        f("cloth_set_proximities", None, [_vp, ctypes.c_int, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp,
                                          ctypes.c_double])
        f("cloth_proximity_forces", None, [_vp, ctypes.c_double, _dp, _dp, _dp, _dp, _dp])
        f("detect_proximities", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _ip, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_int, _ip, _dp, _dp, _dp,
                                               _dp, _dp, _ip])
        f("collision_step", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _ip, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int, _ip])
        f("run_cloths", ctypes.c_double, [ctypes.POINTER(_vp), ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _ip])
        if which == "oracle":
            f("material_new", _vp, [ctypes.c_int, ctypes.c_double, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double])
            f("material_table", None, [_vp, _dp])
        else:
            f("material_new", _vp, [ctypes.c_char_p])
            f("cloth_topology_mismatches", ctypes.c_int, [_vp])

    def fn(self, name, restype, argtypes):
        fobj = getattr(self.lib, self.p + name)
        fobj.restype = restype
        fobj.argtypes = argtypes
        setattr(self, name, fobj)


_LIBS: dict = {}


def lib(which: str = "oracle") -> Lib:
    if which not in _LIBS:
        _LIBS[which] = Lib(which)
    return _LIBS[which]


class Material:
    """A material of the restated oracle (real='float' or 'double') or, with which='ref',
    the reference's own Material built from a written data file."""

    def __init__(self, spec: dict, real: str = "float", which: str = "oracle", workdir: str | None = None):
        self.L = lib(which)
        self.which = which
        self.spec = spec
        if which == "oracle":
            st = _d(np.array(spec["stretching"], np.float64).reshape(24))
            be = _d(np.array(spec["bending"], np.float64).reshape(15))
            self.h = self.L.material_new(0 if real == "float" else 1, spec["density"], _ptr(st, _dp), _ptr(be, _dp),
                                         spec.get("thicken", 1.0), spec.get("density_mult", 1.0),
                                         spec.get("stretching_mult", 1.0), spec.get("bending_mult", 1.0))
        else:
            import json
            path = spec.get("data_file")
            if not path:
                # no data file of the reference's own: write the parameters as one
                wd = workdir or tempfile.mkdtemp(prefix="clothref_")
                path = os.path.join(wd, "material_%d.json" % id(self))
                with open(path, "w") as fh:
                    json.dump({k: spec[k] for k in ("density", "stretching", "bending")}, fh)
            text = json.dumps({"data": path, "thicken": spec.get("thicken", 1.0),
                               "density_mult": spec.get("density_mult", 1.0),
                               "stretching_mult": spec.get("stretching_mult", 1.0),
                               "bending_mult": spec.get("bending_mult", 1.0)})
            self.h = self.L.material_new(text.encode())

    @property
    def density(self) -> float:
        return self.L.material_density(self.h)

    def stretching(self, G3) -> np.ndarray:
        G3 = _d(G3).reshape(-1, 3)
        out = np.zeros((G3.shape[0], 4))
        self.L.material_stretching(self.h, G3.shape[0], _ptr(G3, _dp), _ptr(out, _dp))
        return out

    def bending(self, q5) -> np.ndarray:
        q5 = _d(q5).reshape(-1, 5)
        out = np.zeros(q5.shape[0])
        self.L.material_bending(self.h, q5.shape[0], _ptr(q5, _dp), _ptr(out, _dp))
        return out

    def table(self) -> np.ndarray:
        out = np.zeros(30 * 30 * 30 * 4)
        self.L.material_table(self.h, _ptr(out, _dp))
        return out.reshape(30, 30, 30, 4)

    def __del__(self):
        try:
            self.L.material_free(self.h)
        except Exception:
            pass


class Cloth:
    def __init__(self, sheet: dict, material: Material):
        self.L = material.L
        self.material = material
        x, v, u = _d(sheet["x"]), _d(sheet["v"]), _d(sheet["uv"])
        fx, fu = _i(sheet["fx"]), _i(sheet["fu"])
        self.n = x.shape[0]
        self.nf = fx.shape[0]
        self.h = self.L.cloth_new(material.h, self.n, _ptr(x, _dp), _ptr(v, _dp), u.shape[0], _ptr(u, _dp),
                                  self.nf, _ptr(fx, _ip), _ptr(fu, _ip))
        hn = sheet.get("handles", np.zeros(0, np.int32))
        if len(hn):
            hn = _i(hn)
            pos = _d(x.reshape(-1, 3)[hn])
            self.L.cloth_set_handles(self.h, len(hn), _ptr(hn, _ip), _ptr(pos, _dp))

    def __del__(self):
        try:
            self.L.cloth_free(self.h)
        except Exception:
            pass

    @property
    def n_interior(self) -> int:
        return self.L.cloth_num_interior_edges(self.h)

    def interior_edges(self):
        k = self.n_interior
        nodes = np.zeros((k, 4), np.int32)
        faces = np.zeros((k, 2), np.int32)
        self.L.cloth_interior_edges(self.h, _ptr(nodes, _ip), _ptr(faces, _ip))
        return nodes, faces

    def face_forces(self):
        f = np.zeros((self.nf, 9))
        J = np.zeros((self.nf, 9, 9))
        self.L.cloth_face_forces(self.h, _ptr(f, _dp), _ptr(J, _dp))
        return f, J

    def edge_forces(self):
        k = self.n_interior
        f = np.zeros((k, 12))
        J = np.zeros((k, 12, 12))
        th = np.zeros(k)
        self.L.cloth_edge_forces(self.h, _ptr(f, _dp), _ptr(J, _dp), _ptr(th, _dp))
        return f, J, th

    def assemble(self, params):
        p = _d(params)
        nnzb = self.L.cloth_assemble(self.h, _ptr(p, _dp))
        rp = np.zeros(self.n + 1, np.int32)
        ci = np.zeros(nnzb, np.int32)
        val = np.zeros((nnzb, 3, 3))
        b = np.zeros(3 * self.n)
        self.L.cloth_system(self.h, _ptr(rp, _ip), _ptr(ci, _ip), _ptr(val, _dp), _ptr(b, _dp))
        return rp, ci, val, b

    def solve(self, method=METHOD_LLT, tol=1e-12, max_iter=100000):
        dv = np.zeros(3 * self.n)
        rr = ctypes.c_double(0)
        st = self.L.cloth_solve(self.h, method, tol, max_iter, _ptr(dv, _dp), ctypes.byref(rr))
        if st < -1:
            raise RuntimeError("oracle solve failed (matrix not positive definite)")
        return dv, rr.value

    def step(self, params, method=METHOD_LLT, tol=1e-12, max_iter=100000):
        p = _d(params)
        dv = np.zeros(3 * self.n)
        rr = ctypes.c_double(0)
        st = self.L.cloth_step(self.h, _ptr(p, _dp), method, tol, max_iter, _ptr(dv, _dp), ctypes.byref(rr))
        if st < -1:
            raise RuntimeError("oracle step failed (matrix not positive definite)")
        return dv, rr.value

    def advance(self, dv, dt):
        d = _d(dv)
        self.L.cloth_advance(self.h, _ptr(d, _dp), dt)

    def state(self):
        x = np.zeros(3 * self.n)
        v = np.zeros(3 * self.n)
        self.L.cloth_state(self.h, _ptr(x, _dp), _ptr(v, _dp))
        return x.reshape(-1, 3), v.reshape(-1, 3)

    def set_state(self, x, v):
        x, v = _d(x), _d(v)
        self.L.cloth_set_state(self.h, _ptr(x, _dp), _ptr(v, _dp))

    def masses(self):
        m = np.zeros(self.n)
        self.L.cloth_masses(self.h, _ptr(m, _dp))
        return m

    def normals(self):
        m = np.zeros(3 * self.nf)
        self.L.cloth_normals(self.h, _ptr(m, _dp))
        return m.reshape(-1, 3)

    def set_proximities(self, prox: dict, thickness: float):
        """Proximities of the next steps (Cloth::physicsStep's `proximities`): a dict of arrays
        nodes (n, 4) int (-1: a point outside the cloth), x, v (n, 4, 3) and mass (n, 4) of
        those points, free (n,) bit mask, normal (n, 3), w (n, 4), mu (n,), stiffness (n,)."""
        n = len(prox["mu"])
        self._prox = {k: (_i(v) if k in ("nodes", "free") else _d(v)) for k, v in prox.items()}
        P = self._prox
        self.L.cloth_set_proximities(self.h, n, _ptr(P["nodes"], _ip), _ptr(P["x"], _dp), _ptr(P["v"], _dp),
                                     _ptr(P["mass"], _dp), _ptr(P["free"], _ip), _ptr(P["normal"], _dp),
                                     _ptr(P["w"], _dp), _ptr(P["mu"], _dp), _ptr(P["stiffness"], _dp), thickness)
        self.n_prox = n

    def proximity_forces(self, dt: float):
        """(depth, impulse f, impulse J, friction f, friction J) of every proximity."""
        n = self.n_prox
        fI, fF = np.zeros((n, 12)), np.zeros((n, 12))
        JI, JF = np.zeros((n, 12, 12)), np.zeros((n, 12, 12))
        d = np.zeros(n)
        self.L.cloth_proximity_forces(self.h, dt, _ptr(fI, _dp), _ptr(JI, _dp), _ptr(fF, _dp), _ptr(JF, _dp),
                                      _ptr(d, _dp))
        return d, fI, JI, fF, JF

    def topology_mismatches(self) -> int:
        return self.L.cloth_topology_mismatches(self.h)


def detect_proximities(cloths, groups=None, repulsion_thickness: float = 1e-3, collision_stiffness: float = 1e9,
                       friction: float = 0.6) -> dict:
    """Proximities among the cloths' current states (Simulator::findProximities): node ids
    are scene ids, the cloths' nodes concatenated in the given order; cloths with equal
    groups interact (all of them when groups is None).  Returns a dict of arrays nodes (n, 4),
    normal (n, 3), w (n, 4), mu, stiffness, depth (n,) and kind (n,: 0 node key, 1 edge key,
    2 face key), in the reference's output order."""
    L = cloths[0].L
    arr = (_vp * len(cloths))(*[c.h for c in cloths])
    g = _i(np.zeros(len(cloths)) if groups is None else np.asarray(groups))
    args = (arr, len(cloths), _ptr(g, _ip), repulsion_thickness, collision_stiffness, friction)
    z_i, z_d = np.zeros(1, np.int32), np.zeros(1)
    n = L.detect_proximities(*args, 0, _ptr(z_i, _ip), _ptr(z_d, _dp), _ptr(z_d, _dp), _ptr(z_d, _dp),
                             _ptr(z_d, _dp), _ptr(z_d, _dp), _ptr(z_i, _ip))
    out = {"nodes": np.zeros((n, 4), np.int32), "normal": np.zeros((n, 3)), "w": np.zeros((n, 4)),
           "mu": np.zeros(n), "stiffness": np.zeros(n), "depth": np.zeros(n), "kind": np.zeros(n, np.int32)}
    if n:
        L.detect_proximities(*args, n, _ptr(out["nodes"], _ip), _ptr(out["normal"], _dp), _ptr(out["w"], _dp),
                             _ptr(out["mu"], _dp), _ptr(out["stiffness"], _dp), _ptr(out["depth"], _dp),
                             _ptr(out["kind"], _ip))
    return out


def collision_step(cloths, dt: float, thickness: float = 1e-4, groups=None, max_rounds: int = 0):
    """Simulator::collisionStep over the cloths after their step (positions x0 -> x): resolves
    the impacts, then v = (x - x0) / dt.  Returns (rounds, impacts); rounds -1: unresolved."""
    L = cloths[0].L
    arr = (_vp * len(cloths))(*[c.h for c in cloths])
    g = _i(np.zeros(len(cloths)) if groups is None else np.asarray(groups))
    imp = np.zeros(1, np.int32)
    rounds = L.collision_step(arr, len(cloths), _ptr(g, _ip), thickness, dt, max_rounds, _ptr(imp, _ip))
    return int(rounds), int(imp[0])


def run_cloths(cloths, params_list, steps: int, method: int = METHOD_LLT, threads: int = 1):
    """Steps independent cloths on `threads` host threads; returns (seconds, status)."""
    L = cloths[0].L
    arr = (_vp * len(cloths))(*[c.h for c in cloths])
    p = _d(np.array(params_list, np.float64).reshape(-1))
    st = np.zeros(len(cloths), np.int32)
    sec = L.run_cloths(arr, len(cloths), _ptr(p, _dp), steps, method, threads, _ptr(st, _ip))
    return sec, st


# ---- Handle motions: Transformation, Quaternion and Motion restated in FP32 ----------------
# (Transformation.cu:3-87, Quaternion.cu:3-78, Motion.cu:3-72, JsonHelper.cu).  NumPy float32
# arithmetic is IEEE single precision with no contraction; cos, sin and sqrt are the C library's
# cosf, sinf and sqrtf, as the reference's host code calls them.  A transformation is held as 8
# float32 values: scaling, translation (3), rotation quaternion (s, x, y, z).

_libm = ctypes.CDLL("libm.so.6")
for _fn in ("cosf", "sinf", "sqrtf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]
_f = np.float32


def _transform_identity() -> np.ndarray:
    return np.array([1, 0, 0, 0, 1, 0, 0, 0], np.float32)  # Transformation() (Transformation.cu:3-6)


def transform_from_json(j: dict | None) -> np.ndarray:
    """Transformation(const Json::Value&) (Transformation.cu:8-13): scale (default 1), translate,
    rotate = [degrees, axis x, y, z] -> Quaternion(axis, angle) (Quaternion.cu:7-15)."""
    j = j or {}
    out = _transform_identity()
    out[0] = _f(j.get("scale", 1.0))
    out[1:4] = np.array(j.get("translate", [0.0, 0.0, 0.0]), np.float32)
    r = np.array(j.get("rotate", [0.0, 0.0, 0.0, 0.0]), np.float32)
    angle = _f(np.float64(r[0]) * np.pi / np.float64(_f(180.0)))
    if angle == _f(0.0):
        out[4:8] = [1, 0, 0, 0]
    else:
        half = _f(_f(0.5) * angle)
        ax = r[1:4].astype(np.float32)
        l = _f(_libm.sqrtf(float(_f(_f(ax[0] * ax[0] + ax[1] * ax[1]) + ax[2] * ax[2]))))
        inv = _f(_f(1.0) / l)  # Vector::operator/ multiplies by the reciprocal (Vector.cuh:126-132)
        out[4] = _f(_libm.cosf(float(half)))
        sn = _f(_libm.sinf(float(half)))
        out[5:8] = np.array([_f(sn * _f(ax[k] * inv)) for k in range(3)], np.float32)
    return out


def transform_points(T: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Transformation::applyToPoint (Transformation.cu:82-84): s rotate(p) + t with
    Quaternion::rotate (Quaternion.cu:76-78) p (qs^2 - |qv|^2) + (2 qv)(qv . p) + (2 (qv x p)) qs."""
    T = np.asarray(T, np.float32)
    p = np.asarray(p, np.float32).reshape(-1, 3)
    s, t, qs, qv = T[0], T[1:4], T[4], T[5:8]
    n2 = _f(_f(qv[0] * qv[0] + qv[1] * qv[1]) + qv[2] * qv[2])
    d = ((p[:, 0] * qv[0] + p[:, 1] * qv[1]).astype(np.float32) + (p[:, 2] * qv[2])).astype(np.float32)
    d = ((qv[0] * p[:, 0] + qv[1] * p[:, 1]).astype(np.float32) + qv[2] * p[:, 2]).astype(np.float32)
    cr = np.stack([qv[1] * p[:, 2] - qv[2] * p[:, 1], qv[2] * p[:, 0] - qv[0] * p[:, 2],
                   qv[0] * p[:, 1] - qv[1] * p[:, 0]], 1).astype(np.float32)
    a = p * _f(qs * qs - n2)
    b = (_f(2.0) * qv)[None, :] * d[:, None]
    c = (_f(2.0) * cr) * qs
    r = ((a + b).astype(np.float32) + c).astype(np.float32)
    return ((s * r).astype(np.float32) + t).astype(np.float32)


def _transform_div(T: np.ndarray, s) -> np.ndarray:
    """Transformation::operator/(float) (Transformation.cu:63-69): scaling and the quaternion's
    scalar part divided (Quaternion.cu:58-63), translation and the quaternion's vector part
    multiplied by the reciprocal (Vector::operator/, Vector.cuh:126-132)."""
    s = _f(s)
    inv = _f(_f(1.0) / s)
    out = (T * inv).astype(np.float32)
    out[0] = _f(T[0] / s)
    out[4] = _f(T[4] / s)
    return out


class Motion:
    """Motion (Motion.cu:3-72): keyframes (time, Transformation) with a keyframe at time 0 added
    when the first is later, central-difference tangents (zero at the ends), and per segment the
    cubic a s^3 + b s^2 + c s + d in Transformation arithmetic (componentwise on the 8 values).
    The segment index advances monotonically, as the reference's does."""

    def __init__(self, keyframes: list):
        self.t = [_f(k.get("time", 0.0)) for k in keyframes]
        self.x = [transform_from_json(k.get("transform")) for k in keyframes]
        if self.t[0] > 0:
            self.t.insert(0, _f(0.0))
            self.x.insert(0, _transform_identity())
        n = self.n = len(self.t)
        zero = (_f(0.0) * _transform_identity()).astype(np.float32)
        self.v = [zero] * n
        for i in range(1, n - 1):
            self.v[i] = _transform_div((self.x[i + 1] - self.x[i - 1]).astype(np.float32), _f(self.t[i + 1] - self.t[i - 1]))
        self.index = 0
        self._coefficients()

    def _coefficients(self):
        i = self.index
        dt = _f(self.t[i + 1] - self.t[i])
        dx = (self.x[i + 1] - self.x[i]).astype(np.float32)
        v0, v1 = self.v[i], self.v[i + 1]
        self.a = ((dt * (v1 + v0).astype(np.float32)).astype(np.float32) - (_f(2.0) * dx)).astype(np.float32)
        self.b = ((_f(3.0) * dx) - (dt * (v1 + (_f(2.0) * v0)).astype(np.float32)).astype(np.float32)).astype(np.float32)
        self.c = (dt * v0).astype(np.float32)
        self.d = self.x[i]

    def transform(self, time: float) -> np.ndarray:
        time = _f(time)
        moved = False
        while self.index < self.n - 1 and self.t[self.index + 1] < time:
            self.index += 1
            moved = True
        if self.index == self.n - 1:
            return self.x[self.n - 1].copy()
        if moved:
            self._coefficients()
        s = _f(_f(time - self.t[self.index]) / _f(self.t[self.index + 1] - self.t[self.index]))
        s2 = _f(s * s)
        s3 = _f(s * s2)
        return ((((self.a * s3).astype(np.float32) + (self.b * s2)).astype(np.float32) + (self.c * s)).astype(np.float32)
                + self.d).astype(np.float32)


def ref_transform_points(transform_json: dict, p: np.ndarray) -> np.ndarray:
    """The reference's own Transformation(json).applyToPoint (the adapter library)."""
    import json

    L = lib("ref")
    fn = L.lib.ref_transform_points
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, _dp, _dp]
    p = _d(p).reshape(-1, 3)
    out = np.zeros_like(p)
    fn(json.dumps(transform_json).encode(), p.shape[0], _ptr(p, _dp), _ptr(out, _dp))
    return out


def ref_motion_points(keyframes: list, times, p: np.ndarray) -> np.ndarray:
    """The reference's own Motion(json).computeTransformation(t).applyToPoint at each time."""
    import json

    L = lib("ref")
    fn = L.lib.ref_motion_points
    fn.argtypes = [ctypes.c_char_p, ctypes.c_int, _dp, ctypes.c_int, _dp, _dp]
    p = _d(p).reshape(-1, 3)
    ts = _d(times)
    out = np.zeros((len(ts), p.shape[0], 3))
    fn(json.dumps(keyframes).encode(), len(ts), _ptr(ts, _dp), p.shape[0], _ptr(p, _dp), _ptr(out, _dp))
    return out
