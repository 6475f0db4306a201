"""Seeded synthetic cloth scenes for the implicit-step workloads.

Every scene is a list of sheets.  A sheet is a dict of NumPy arrays in the layout the
C ABI takes (``cs_load_batch``): node positions ``x`` (N,3) float32, velocities ``v``
(N,3), uv rest coordinates ``uv`` (U,2), triangle corners as node indices ``fx`` (F,3)
int32 and uv-vertex indices ``fu`` (F,3), handle node indices ``handles`` and the
material and wind parameters.  Triangles are counter-clockwise in the uv plane, so
every interior edge has one adjacent face on each side, as ``Edge::initialize``
expects (Edge.cu:13-31).

Material parameters follow the reference's material JSON plus the cloth's
``materials`` multipliers (Material.cu:3-41): ``density``, six ``stretching`` rows of
four values, 3x5 ``bending`` samples, ``thicken`` and ``density_mult`` /
``stretching_mult`` / ``bending_mult``.  Wind follows Wind.cu:3-7 (density defaults to
1, drag and velocity to 0).  No public dataset is involved: all inputs are generated
here from the seed.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

GRAVITY = (0.0, -9.8, 0.0)


def isotropic_material(stiffness: float, bending: float, density: float = 0.2) -> dict:
    """Material whose six stretching rows are all [E, 0, E, E] and whose 15 bending
    samples are all equal.  The reference doubles table values internally
    (Material.cu:82) exactly like the GPU path, so the rows are the file values."""
    return {
        "density": float(density),
        "stretching": [[float(stiffness), 0.0, float(stiffness), float(stiffness)]] * 6,
        "bending": [[float(bending)] * 5] * 3,
        "thicken": 1.0,
        "density_mult": 1.0,
        "stretching_mult": 1.0,
        "bending_mult": 1.0,
    }


def scaled_unit_material(stiffness: float, bending: float, density: float = 0.2) -> dict:
    """A unit base file ([1,0,1,1] rows, bending 1) scaled through the cloth's
    stretching_mult / bending_mult, as the batched workloads specify."""
    m = isotropic_material(1.0, 1.0, density)
    m["stretching_mult"] = float(stiffness)
    m["bending_mult"] = float(bending)
    return m


def no_wind() -> dict:
    return {"density": 1.0, "drag": 0.0, "velocity": [0.0, 0.0, 0.0]}


def grid_sheet(nq: int, size: float = 1.0, *, rng: np.random.Generator, z_noise: float = 0.0,
               flip_prob: float | None = None, jitter: float = 0.0, vel_sigma: float = 0.0) -> dict:
    """A size x size sheet of nq x nq quads in the x-y plane, hanging along -y.

    Node (i, j) is column i, row j (y grows with j), numbered j*(nq+1)+i.  Each quad is
    split along alternating diagonals ((i+j) even: lower-left to upper-right), or, with
    ``flip_prob``, along a diagonal drawn per quad.  ``jitter`` moves interior nodes in
    the plane, in x and in uv alike, by a displacement drawn uniformly from the disk of
    radius jitter*h.  Up to 0.35 no triangle inverts (three nodes close at most 2*jitter*h
    of a right triangle's h/sqrt(2) altitude); independent per-axis offsets of 0.3 h would
    move a node 0.42 h along a diagonal and invert some triangles.
    """
    n = nq + 1
    h = size / nq
    jj, ii = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    u = np.stack([ii * h, jj * h], axis=-1).reshape(-1, 2).astype(np.float64)
    if jitter > 0.0:
        interior = ((ii > 0) & (ii < nq) & (jj > 0) & (jj < nq)).reshape(-1)
        rad = jitter * h * np.sqrt(rng.uniform(0.0, 1.0, size=n * n))
        ang = rng.uniform(0.0, 2.0 * np.pi, size=n * n)
        d = np.stack([rad * np.cos(ang), rad * np.sin(ang)], axis=-1)
        u[interior] += d[interior]
    x = np.zeros((n * n, 3), np.float64)
    x[:, :2] = u
    if z_noise > 0.0:
        x[:, 2] = rng.normal(0.0, z_noise, size=n * n)
    qi, qj = np.meshgrid(np.arange(nq), np.arange(nq), indexing="ij")
    qi = qi.T.reshape(-1)
    qj = qj.T.reshape(-1)
    a = qj * n + qi
    b = a + 1
    c = a + n + 1
    dd = a + n
    if flip_prob is None:
        main = ((qi + qj) % 2) == 0
    else:
        main = rng.random(nq * nq) >= flip_prob
    t1 = np.where(main[:, None], np.stack([a, b, c], 1), np.stack([a, b, dd], 1))
    t2 = np.where(main[:, None], np.stack([a, c, dd], 1), np.stack([b, c, dd], 1))
    f = np.stack([t1, t2], 1).reshape(-1, 3).astype(np.int32)
    v = np.zeros((n * n, 3), np.float64)
    if vel_sigma > 0.0:
        v = rng.normal(0.0, vel_sigma, size=(n * n, 3))
    return {
        "nq": nq,
        "x": x.astype(np.float32),
        "v": v.astype(np.float32),
        "uv": u.astype(np.float32),
        "fx": f,
        "fu": f.copy(),
    }


def top_edge(nq: int) -> np.ndarray:
    n = nq + 1
    return (nq * n + np.arange(n)).astype(np.int32)


def corners(nq: int) -> np.ndarray:
    n = nq + 1
    return np.array([nq * n, nq * n + nq, 0, nq], np.int32)  # top-left, top-right, bottom-left, bottom-right


@dataclass
class Scene:
    name: str
    sheets: list
    dt: float
    steps: int
    gravity: tuple = GRAVITY
    handle_stiffness: float = 1e3  # Magic.cu:6
    tol: float = 1e-6
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(sum(s["x"].shape[0] for s in self.sheets))

    @property
    def n_faces(self) -> int:
        return int(sum(s["fx"].shape[0] for s in self.sheets))


def hang(nq: int = 32, seed: int = 0) -> Scene:
    """Plain implicit step: 1 m sheet of nq x nq quads, top two corners pinned, z noise
    N(0, 1 mm), isotropic 50 N/m, bending 1e-5 N m, density 0.2, dt 1/100, 200 steps."""
    rng = np.random.default_rng(seed)
    s = grid_sheet(nq, rng=rng, z_noise=1e-3)
    s["handles"] = corners(nq)[:2].copy()
    s["material"] = isotropic_material(50.0, 1e-5)
    s["wind"] = no_wind()
    return Scene("hang32" if nq == 32 else f"hang{nq}", [s], dt=1.0 / 100, steps=200)


def precision_sheet(nq: int = 256, seed: int = 0) -> Scene:
    """Precision study: nq x nq sheet, top edge pinned, per-node velocities N(0, 0.1),
    isotropic 200 N/m, bending 1e-4, density 0.2, dt 1/200, one step."""
    rng = np.random.default_rng(seed)
    s = grid_sheet(nq, rng=rng, vel_sigma=0.1)
    s["handles"] = top_edge(nq)
    s["material"] = isotropic_material(200.0, 1e-4)
    s["wind"] = no_wind()
    return Scene(f"precision{nq}", [s], dt=1.0 / 200, steps=1, tol=1e-6)


def uneven_batch(n_sheets: int = 512, seed: int = 0, nq_range=(16, 128)) -> Scene:
    """Batched uneven sheets: side nq log-uniform in nq_range, 1-4 corners pinned,
    stretching log-U[10, 500] N/m and bending log-U[1e-6, 1e-3] N m through the
    multipliers of a unit base material, density 0.2, dt 1/100, 100 steps."""
    rng = np.random.default_rng(seed)
    sheets = []
    for _ in range(n_sheets):
        nq = int(round(math.exp(rng.uniform(math.log(nq_range[0]), math.log(nq_range[1])))))
        s = grid_sheet(nq, rng=rng, z_noise=1e-3)
        k = int(rng.integers(1, 5))
        s["handles"] = np.sort(rng.choice(corners(nq), size=k, replace=False)).astype(np.int32)
        E = math.exp(rng.uniform(math.log(10.0), math.log(500.0)))
        B = math.exp(rng.uniform(math.log(1e-6), math.log(1e-3)))
        s["material"] = scaled_unit_material(E, B)
        s["wind"] = no_wind()
        sheets.append(s)
    return Scene("uneven512" if n_sheets == 512 else f"uneven{n_sheets}", sheets, dt=1.0 / 100, steps=100)


def windy_batch(n_sheets: int = 1024, nq: int = 64, seed: int = 0) -> Scene:
    """Learned-warm-start workload: n_sheets sheets of nq x nq quads, top edge pinned,
    per-sheet horizontal wind (direction U[0, 2pi), speed U(0, 10) m/s, drag 1), materials
    as in the uneven batch, dt 1/100."""
    rng = np.random.default_rng(seed)
    base = grid_sheet(nq, rng=rng)
    sheets = []
    for _ in range(n_sheets):
        s = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in base.items()}
        s["x"] = s["x"].copy()
        s["x"][:, 2] = rng.normal(0.0, 1e-3, size=s["x"].shape[0]).astype(np.float32)
        s["handles"] = top_edge(nq)
        E = math.exp(rng.uniform(math.log(10.0), math.log(500.0)))
        B = math.exp(rng.uniform(math.log(1e-6), math.log(1e-3)))
        s["material"] = scaled_unit_material(E, B)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        speed = rng.uniform(0.0, 10.0)
        s["wind"] = {"density": 1.0, "drag": 1.0, "velocity": [speed * math.cos(phi), 0.0, speed * math.sin(phi)]}
        sheets.append(s)
    return Scene(f"windy{n_sheets}x{nq}", sheets, dt=1.0 / 100, steps=200)


def large_irregular(nq: int = 1000, seed: int = 0) -> Scene:
    """Large irregular sheet: 2 m x 2 m, nq x nq quads, interior nodes jittered by
    +-0.3 h in x and uv, each quad's diagonal flipped with p = 0.5, top edge pinned,
    wind (0, 0, 5) m/s with drag 1, isotropic 100 N/m, bending 1e-5, dt 1/200, 50 steps.
    The sheet starts flat: out-of-plane noise of the hanging sheets' 1 mm would strain a
    2 mm spacing by ~25 % and crumple it."""
    rng = np.random.default_rng(seed)
    s = grid_sheet(nq, size=2.0, rng=rng, flip_prob=0.5, jitter=0.3)
    s["handles"] = top_edge(nq)
    s["material"] = isotropic_material(100.0, 1e-5)
    s["wind"] = {"density": 1.0, "drag": 1.0, "velocity": [0.0, 0.0, 5.0]}
    return Scene(f"irregular{nq}", [s], dt=1.0 / 200, steps=50)


def synthetic_proximities(sheet: dict, rng: np.random.Generator, n_vf: int = 6, n_ee: int = 4, n_ext: int = 4,
                          stiffness: float = 1e4, thickness: float = 5e-3, node_off: int = 0) -> dict:
    """Seeded proximity records of the kind Cloth::physicsStep receives (Proximity.cu:5-24):
    vertex-face pairs inside the sheet (weights 1 and minus the barycentric weights of the
    face point, the face normal), edge-edge pairs (weights 1 - s, s, -(1 - t), -t, the
    normalised cross product of the edges), and external points (an obstacle-like point
    near a face: node -1 with its own position, velocity and mass, not free).  Stiffness is
    `stiffness` times the smaller rest area, as the constructors scale it.  Node ids are
    offset by `node_off` (for a sheet inside a batch)."""
    x = sheet["x"].astype(np.float64)
    v = sheet["v"].astype(np.float64)
    fx = sheet["fx"]
    nn = x.shape[0]
    u = sheet["uv"].astype(np.float64)
    e1 = u[fx[:, 1]] - u[fx[:, 0]]
    e2 = u[fx[:, 2]] - u[fx[:, 0]]
    farea = 0.5 * np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0])
    recs = {k: [] for k in ("nodes", "x", "v", "mass", "free", "normal", "w", "mu", "stiffness")}

    def face_normal(f):
        a, b_, c = x[fx[f, 0]], x[fx[f, 1]], x[fx[f, 2]]
        n = np.cross(b_ - a, c - a)
        return n / np.linalg.norm(n)

    def add(nodes, w, n, mu, k, xe=None, ve=None, me=None, free=0):
        recs["nodes"].append([(i + node_off) if i >= 0 else -1 for i in nodes])
        recs["x"].append(xe if xe is not None else np.zeros((4, 3)))
        recs["v"].append(ve if ve is not None else np.zeros((4, 3)))
        recs["mass"].append(me if me is not None else np.ones(4))
        recs["free"].append(free)
        recs["normal"].append(n)
        recs["w"].append(w)
        recs["mu"].append(mu)
        recs["stiffness"].append(k)

    for _ in range(n_vf):
        f = int(rng.integers(len(fx)))
        i = int(rng.integers(nn))
        while i in fx[f]:
            i = int(rng.integers(nn))
        bc = rng.dirichlet(np.ones(3))
        add([i, *fx[f]], [1.0, -bc[0], -bc[1], -bc[2]], face_normal(f), rng.uniform(0.1, 0.6),
            stiffness * farea[f] * rng.uniform(0.5, 1.0))
    for _ in range(n_ee):
        f0, f1 = rng.choice(len(fx), 2, replace=False)
        p0, p1 = fx[f0, 0], fx[f0, 1]
        q0, q1 = fx[f1, 1], fx[f1, 2]
        if len({p0, p1, q0, q1}) < 4:
            continue
        n = np.cross(x[p1] - x[p0], x[q1] - x[q0])
        n = n / np.linalg.norm(n) if np.linalg.norm(n) > 1e-12 else np.array([0.0, 0.0, 1.0])
        s_, t_ = rng.uniform(0, 1, 2)
        add([p0, p1, q0, q1], [1 - s_, s_, -(1 - t_), -t_], n, rng.uniform(0.1, 0.6),
            stiffness * min(farea[f0], farea[f1]))
    for _ in range(n_ext):
        f = int(rng.integers(len(fx)))
        bc = rng.dirichlet(np.ones(3))
        n = face_normal(f)
        pt = bc @ x[fx[f]] + n * rng.uniform(0.0, thickness)
        xe = np.zeros((4, 3))
        ve = np.zeros((4, 3))
        xe[0] = pt
        ve[0] = rng.normal(0, 0.05, 3)
        me = np.ones(4)
        add([-1, *fx[f]], [1.0, -bc[0], -bc[1], -bc[2]], n, rng.uniform(0.1, 0.6), stiffness * farea[f], xe, ve, me)
    return {k: np.asarray(vv, dtype=np.int32 if k in ("nodes", "free") else np.float64) for k, vv in recs.items()}


def folded_sheet(nq: int = 16, gap: float = 1.5e-3, seed: int = 0) -> Scene:
    """Self-contact: a 1 m sheet of nq x nq quads (nq even) folded over itself along x = 0.5,
    the upper half `gap` above the lower one and shifted in-plane by (0.3 h, 0.2 h) so its
    nodes project inside the lower faces; z noise N(0, 0.1 mm).  Crease nodes stay on the
    lower layer; the lower edge at x = 0 is pinned.  dt 1/100."""
    assert nq % 2 == 0
    rng = np.random.default_rng(seed)
    s = grid_sheet(nq, rng=rng)
    h = 1.0 / nq
    x = s["x"].astype(np.float64)
    upper = x[:, 0] > 0.5 + 1e-9
    x[upper, 0] = 1.0 - x[upper, 0] + 0.3 * h
    x[upper, 1] += 0.2 * h
    x[upper, 2] = gap
    x[:, 2] += rng.normal(0.0, 1e-4, size=x.shape[0])
    s["x"] = x.astype(np.float32)
    n = nq + 1
    s["handles"] = (np.arange(n) * n).astype(np.int32)  # column x = 0
    s["material"] = isotropic_material(50.0, 1e-5)
    s["wind"] = no_wind()
    return Scene(f"folded{nq}", [s], dt=1.0 / 100, steps=20, meta={"gap": gap})


def stacked_sheets(nq: int = 16, gap: float = 1.5e-3, n_layers: int = 2, seed: int = 0) -> Scene:
    """Cross-sheet contact: n_layers sheets of nq x nq quads stacked `gap` apart, each layer
    shifted in-plane by (0.3 h, 0.2 h) from the one below, z noise N(0, 0.1 mm), top edges
    pinned.  dt 1/100."""
    rng = np.random.default_rng(seed)
    sheets = []
    h = 1.0 / nq
    for k in range(n_layers):
        s = grid_sheet(nq, rng=rng)
        x = s["x"].astype(np.float64)
        x[:, 0] += 0.3 * h * k
        x[:, 1] += 0.2 * h * k
        x[:, 2] = gap * k + rng.normal(0.0, 1e-4, size=x.shape[0])
        s["x"] = x.astype(np.float32)
        s["handles"] = top_edge(nq)
        s["material"] = isotropic_material(50.0, 1e-5)
        s["wind"] = no_wind()
        sheets.append(s)
    return Scene(f"stacked{n_layers}x{nq}", sheets, dt=1.0 / 100, steps=20, meta={"gap": gap})


WORKLOADS = {
    "hang32": lambda seed=0: hang(32, seed),
    "precision256": lambda seed=0: precision_sheet(256, seed),
    "uneven512": lambda seed=0: uneven_batch(512, seed),
    "windy1024x64": lambda seed=0: windy_batch(1024, 64, seed),
    "irregular1000": lambda seed=0: large_irregular(1000, seed),
}


def write_material_file(material: dict, directory: str, name: str) -> str:
    """Writes the material's data file (density, stretching, bending) in the reference's
    format (materials/*.json) and returns its path."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, name + ".json")
    data = {k: material[k] for k in ("density", "stretching", "bending")}
    with open(path, "w") as fh:
        json.dump(data, fh)
    return path


def material_spec_json(material: dict, data_path: str) -> str:
    """The cloth's "materials" object as the reference reads it (Material.cu:4-8)."""
    return json.dumps({
        "data": data_path,
        "thicken": material.get("thicken", 1.0),
        "density_mult": material.get("density_mult", 1.0),
        "stretching_mult": material.get("stretching_mult", 1.0),
        "bending_mult": material.get("bending_mult", 1.0),
    })


def write_obj(sheet: dict, path: str) -> None:
    """Writes a sheet in the reference's OBJ dialect (v, nv, vt, f x/u; Mesh.cu:454-507)."""
    with open(path, "w") as fh:
        for p, q in zip(sheet["x"], sheet["v"]):
            fh.write("v %.9g %.9g %.9g\n" % tuple(p))
            fh.write("nv %.9g %.9g %.9g\n" % tuple(q))
        for t in sheet["uv"]:
            fh.write("vt %.9g %.9g\n" % tuple(t))
        for a, b in zip(sheet["fx"], sheet["fu"]):
            fh.write("f %d/%d %d/%d %d/%d\n" % (a[0] + 1, b[0] + 1, a[1] + 1, b[1] + 1, a[2] + 1, b[2] + 1))


def step_params(scene: Scene, sheet: dict) -> list:
    """Packed parameters [dt, g(3), wind density, drag, wind velocity(3), handle stiffness]."""
    w = sheet["wind"]
    return [scene.dt, *scene.gravity, w["density"], w["drag"], *w["velocity"], scene.handle_stiffness]


def write_scene(scene: Scene, directory: str, frames: int = 2, solver: dict | None = None) -> str:
    """Writes a scene in the reference's format: one OBJ per sheet, its material data file,
    and a config JSON with the reference's keys (frame_time, frame_steps, end_frame, gravity,
    wind, magic, cloths[mesh, materials], handles[cloth, nodes], disable) -- plus the
    per-cloth "wind" and the "solver" object, extensions the reference ignores.  Returns the
    config path."""
    os.makedirs(directory, exist_ok=True)
    cloths, handles = [], []
    for i, s in enumerate(scene.sheets):
        mesh = os.path.join(directory, f"sheet{i}.obj")
        write_obj(s, mesh)
        data = write_material_file(s["material"], directory, f"material{i}")
        m = s["material"]
        cloths.append({"mesh": mesh, "materials": {"data": data, "thicken": m.get("thicken", 1.0),
                                                   "density_mult": m.get("density_mult", 1.0),
                                                   "stretching_mult": m.get("stretching_mult", 1.0),
                                                   "bending_mult": m.get("bending_mult", 1.0)},
                       "wind": s["wind"]})
        if len(s.get("handles", [])):
            handles.append({"cloth": i, "nodes": [int(n) for n in s["handles"]]})
    config = {
        "frame_time": scene.dt * 4, "frame_steps": 4, "end_frame": frames,
        "gravity": list(scene.gravity), "magic": {"handle_stiffness": scene.handle_stiffness},
        "cloths": cloths, "handles": handles, "disable": ["remeshing"],
    }
    if solver:
        config["solver"] = solver
    path = os.path.join(directory, "config.json")
    with open(path, "w") as fh:
        fh.write("// generated scene\n" + json.dumps(config, indent=2))
    return path
