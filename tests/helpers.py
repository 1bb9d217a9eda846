"""Shared test helpers: golden fixtures and oracle runs."""
import glob
import os

import numpy as np

from oracle import py as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RHO_W = 0.334


def golden_cases(prefix=""):
    """Histogram/intensity fixtures (grid excluded-volume, fit and calculator fixtures are listed by
    grid_cases, fit_cases and calc_cases; the multi-step partial-manager and hydration fixtures belong to their own tests)."""
    return sorted(n for n in (os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))
                  if not n.startswith(("gridexv_", "fit_", "calc_", "partial_", "hydrate_", "fullsize_")))


def grid_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "gridexv_*.npz")))


def fit_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "fit_*.npz")))


FIT_KIND = {"ffavg": 0, "ffexplicit": 1, "ffgrid": 2, "mt": 3}


def calc_cases():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "calc_*.npz")))


def calc_inputs(g):
    """Point sets and the job list [(a, b or None, scaling, merge_id)] of a calculator fixture."""
    off = g["offsets"]
    sets = [g["points"][off[k]:off[k + 1]] for k in range(len(off) - 1)]
    jobs = [(int(a), None if b < 0 else int(b), int(sc), int(m)) for a, b, sc, m in g["jobs"]]
    return sets, jobs


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def simple_exv_weights(w, volume, n_atoms):
    """CompactCoordinatesTemplate::implicit_excluded_volume: w += -(rho_w * V / N), in double, stored as float."""
    return (np.asarray(w, np.float32).astype(np.float64) - RHO_W * volume / n_atoms).astype(np.float32)


def oracle_for(g):
    """Run the C restatement on a golden fixture's inputs."""
    mgr = str(g["manager"])
    bw = float(g["bin_width"])
    atoms, waters = g["atoms"], g["waters"]
    if mgr == "mt":
        w = g["w"]
        if bool(g["simple_exv"]):
            w = simple_exv_weights(w, float(g["volume"]), len(atoms))
        A = O.pack_points(atoms, w, False)
        W = O.pack_points(waters, g["ww"], False)
        return O.hist_simple(A, W, bw, 8000)
    kind = {"ffavg": 0, "ffexplicit": 1, "ffgrid": 2}[mgr]
    A = O.pack_points(atoms, g["ff"], True)
    W = O.pack_points(waters, np.ones(len(waters), np.int32), True)
    X = O.pack_points(g["exv"], np.zeros(len(g["exv"]), np.int32), True)
    z = float(g["volume"]) * RHO_W / len(atoms)
    return O.hist_ff(kind, A, W, X if kind == 2 else None, bw, 8000, z)


def input_digest(m) -> str:
    """SHA-256 over a molecule's float64 inputs (atoms, form-factor types, waters, dummies, volume): the
    full-size fixtures store it so that regenerating their inputs from the seed is checked to be exact."""
    import hashlib

    h = hashlib.sha256()
    for a in (m.atoms, m.ff_types.astype(np.int64), m.waters, m.exv if m.exv is not None else np.zeros((0, 3))):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(np.float64(m.volume).tobytes())
    return h.hexdigest()
