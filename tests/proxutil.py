"""Helpers shared by the proximity tests: the per-cloth view of batch-wide proximities that
the oracle's cloths receive (Cloth::physicsStep marks nodes outside the cloth with index -1,
Cloth.cu:171-192)."""
import numpy as np

import pyoracle


def offsets(scene):
    return np.cumsum([0] + [s["x"].shape[0] for s in scene.sheets]).astype(int)


def full_records(prox):
    """Adds zero outside-point fields to a dict of detected proximities."""
    n = len(prox["mu"])
    out = dict(prox)
    out.setdefault("x", np.zeros((n, 4, 3)))
    out.setdefault("v", np.zeros((n, 4, 3)))
    out.setdefault("mass", np.ones((n, 4)))
    out.setdefault("free", np.zeros(n, np.int32))
    return {k: out[k] for k in ("nodes", "x", "v", "mass", "free", "normal", "w", "mu", "stiffness")}


def oracle_proximities(prox, k, offs, x, v, mass):
    """The proximities sheet k's cloth receives: its nodes local, every other batch node -1
    with the state it has at the start of the step (a free point, with its lumped mass)."""
    lo, hi = offs[k], offs[k + 1]
    sel = [p for p in range(len(prox["mu"])) if np.any((prox["nodes"][p] >= lo) & (prox["nodes"][p] < hi))]
    out = {key: np.array(val[sel]) for key, val in prox.items()}
    for r, p in enumerate(sel):
        for i in range(4):
            nd = int(prox["nodes"][p, i])
            if lo <= nd < hi:
                out["nodes"][r, i] = nd - lo
            elif nd >= 0:
                out["nodes"][r, i] = -1
                out["x"][r, i] = x[nd]
                out["v"][r, i] = v[nd]
                out["mass"][r, i] = mass[nd]
                out["free"][r] |= 1 << i
    return out


def touched_sheets(prox, offs):
    nodes = prox["nodes"][prox["nodes"] >= 0]
    return sorted({int(np.searchsorted(offs, nd, side="right") - 1) for nd in nodes})


def set_oracle_proximities(cloths, prox, offs, thickness, x=None, v=None):
    """Hands each oracle cloth its view of the batch proximities; x, v default to the cloths'
    own current states."""
    if x is None:
        x = np.concatenate([c.state()[0] for c in cloths])
        v = np.concatenate([c.state()[1] for c in cloths])
    mass = np.concatenate([c.masses() for c in cloths])
    prox = full_records(prox)
    for k in range(len(cloths)):
        cloths[k].set_proximities(oracle_proximities(prox, k, offs, x, v, mass), thickness)
