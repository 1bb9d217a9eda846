"""Regenerate the golden fixtures from the reference compiled from its own sources.

Run (needs oracle/_ref/libausaxs_ref.so, i.e. a machine where the reference sources were
available to ``make -C oracle``):

    python tests/golden/make_golden.py

Each fixture stores the inputs (coordinates as float64, form-factor types, weights, waters,
exv dummies, volume, settings) and the reference's outputs: the raw histograms of
calculate_all(), the distance axes, and debye_transform() with its partial profiles on the
reference's default q axis.  Cases:

* ``cube_*``  : the reference's SimpleCube known-answer structure (tests/feature/hist/hist_test_helper.h:87-162)
                for every manager;
* ``random_*``: seeded random molecules (ragged sizes, all four elements, non-default bin width);
* ``pdb_*``   : the proteins 2epe and 6lyz from the reference's own test files, read by the
                reference's reader (united-atom form-factor types);
* ``gridexv_*``: RawGridExv dummies and grid volumes;
* ``fit_*``   : SmartFitter::fit with the Golden minimiser over one parameter, on synthetic data on
                the model's own q axis;
* ``calc_*``  : SimpleCalculator job lists (scaling factors, merge ids);
* ``partial_*``: PartialHistogramManagerMT over a multi-body molecule, initially and after rigid moves;
* ``hydrate_*``: Molecule::generate_new_hydration() (RadialHydration) with seeded noise tables, on a
                fresh grid and after rigid moves.

Full-size fixtures (``python tests/golden/make_golden.py fullsize``; minutes of reference CPU time):

* ``fullsize_cfg1``: the 50,000-atom globule with 10,000 waters and its 1 A grid dummies
                (HistogramManagerMTFFGrid, 0.1 A bins) and ``fullsize_cfg2``: the 500,000-atom icosahedral
                shell with 60,000 waters (HistogramManagerMTFFAvg, 0.1 A bins);
* ``fullsize_cfg3``: 8 structures of the seeded 256-structure batch, spread over its size range
                (HistogramManagerMTFFAvg, 0.25 A bins).
Their inputs are not stored: ausaxs_b200.synth regenerates them from the seed, and a SHA-256 digest of
the float64 inputs is stored to prove the regeneration identical.  Stored: the reference's raw
counts by form-factor type, its distance axes, and I(q) at the workload's q grid from the oracle's
generalised-q transform applied to the reference's histograms.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import py as O  # noqa: E402
from tests.helpers import input_digest  # noqa: E402

REF_ROOT = os.environ.get("AUSAXS_REFERENCE", "/root/reference")  # reference checkout (read-only)

CUBE = np.array([[-1, -1, -1], [-1, 1, -1], [1, -1, -1], [1, 1, -1], [-1, -1, 1], [-1, 1, 1], [1, -1, 1], [1, 1, 1]], float)


def run_case(name, atoms, ff, w, waters, ww, exv, volume, bin_width, manager, cw=1.0, cx=1.0, crho=1.0, dwa=0.0, dwx=0.0,
             simple_exv=False):
    O.ref_set_axes(bin_width, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(simple_exv)
    m = O.RefMolecule(atoms, w, ff, waters, ww, volume=volume)
    m.set_manager(manager, exv_xyz=exv if manager == "ffgrid" else None)
    h = m.calculate()
    out = dict(atoms=atoms, ff=ff.astype(np.int32), w=w, waters=waters, ww=ww, exv=exv, volume=volume,
               bin_width=bin_width, manager=manager, params=np.array([cw, cx, crho, dwa, dwx]),
               simple_exv=simple_exv)
    tot, d = h.total()
    out["tot"], out["d_axis"] = tot, d
    if manager in ("mt", "single"):
        out["aa"], out["aw"], out["ww_h"] = h.simple()
    else:
        out["aa"], out["aw"], out["ww_h"] = h.ff()
        if manager == "ffgrid":
            ax, xx = h.grid_axes()
            out["d_axis_ax"], out["d_axis_xx"] = ax[: len(d)], xx[: len(d)]
    q, I, prof, _ = h.debye(cw, cx, crho, dwa, dwx)
    out["q"], out["Iq"], out["profiles"] = q, I, prof
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "bins", len(d), "I" if "Iq" in out else "")


def grid_case(name, atoms, ff, waters):
    d, vol = O.ref_grid_exv(atoms, ff, waters)
    assert np.all(d == np.round(d)), "dummies of a 1 A grid with integer bounds sit at integer coordinates"
    np.savez_compressed(os.path.join(HERE, name + ".npz"), atoms=atoms, ff=np.asarray(ff, np.int32), waters=waters,
                        dummies=d.astype(np.int32), volume=vol, manager="gridexv")
    print(name, "dummies", len(d), "volume", vol)


FIT_PARAMS = ("cw", "cx", "crho", "dw_atomic", "dw_exv")


def fit_case(name, atoms, ff, w, waters, ww, exv, volume, bin_width, manager, param, truth, seed):
    """SmartFitter::fit (Golden over one parameter) on synthetic data: the model on its own q axis at
    the true parameter value, scaled, offset and with 1 % Gaussian noise (a separate seeded stream)."""
    O.ref_set_axes(bin_width, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(False)
    m = O.RefMolecule(atoms, w, ff, waters, ww, volume=volume)
    m.set_manager(manager, exv_xyz=exv if manager == "ffgrid" else None)
    h = m.calculate()
    base = [1.0, 1.0, 1.0, 0.0, 0.0]
    true = list(base)
    true[param] = truth
    q, I, _, _ = h.debye(*true)
    r = np.random.default_rng(seed)
    y0 = 2.5 * I + 0.002 * np.abs(I).max()
    sigma = 0.01 * np.abs(y0) + 1e-6 * np.abs(y0).max()
    y = y0 + sigma * r.standard_normal(len(q))
    h.debye(*base)  # the histogram's free parameters back at their defaults before fitting
    fit = h.fit(param, q, y, sigma)
    out = dict(atoms=atoms, ff=ff.astype(np.int32), w=w, waters=waters, ww=ww, exv=exv, volume=volume,
               bin_width=bin_width, manager=manager, simple_exv=False, fit_param=param, fit_truth=truth,
               fit_base=np.array(base), q=q, y=y, sigma=sigma, fit_out=np.array(fit[:4] + (float(fit[4]),)))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, FIT_PARAMS[param], "truth", truth, "fit", fit)


def calc_case(name, sets, jobs, bin_width):
    """hist::distance_calculator::SimpleCalculator<true, false> on a job list (self and cross jobs with
    scaling factors and merge ids, as SymmetryManagerMT issues them)."""
    O.ref_set_axes(bin_width, 8000, 1e-4, 0.5)
    res = O.ref_calculator(sets, jobs)
    keys = sorted(res)
    last = max(int(np.max(np.nonzero(np.any(np.stack(res[k]) != 0, axis=0))[0])) for k in keys) + 1
    out = dict(points=np.concatenate(sets).astype(np.float32), offsets=np.cumsum([0] + [len(x) for x in sets]),
               jobs=np.array([(a, -1 if b is None else b, sc, m) for a, b, sc, m in jobs], np.int32),
               bin_width=bin_width, manager="calculator", keys=np.array(keys, np.int32),
               results=np.stack([np.stack(res[k])[:, :last] for k in keys]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "results", len(keys), "bins", last)


def rotation(axis, angle):
    axis = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K


def partial_case(name, bodies, ws, waters, ww, moves, bin_width):
    """PartialHistogramManagerMT over a multi-body molecule: calculate_all() initially and after each
    rigid move (body, R, t); per step the bodies' and the waters' coordinates (the waters belong to a
    body and move with it) and the composite histogram."""
    O.ref_set_axes(bin_width, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(False)
    xyz = np.concatenate(bodies)
    m = O.RefMolecule(xyz, np.concatenate(ws), np.full(len(xyz), 3), waters, ww, body_sizes=[len(b) for b in bodies],
                      volume=18.0 * len(xyz))
    m.set_manager("partial")
    out = dict(weights=np.concatenate(ws), body_sizes=np.array([len(b) for b in bodies], np.int32), waters=waters, ww=ww,
               bin_width=bin_width, manager="partial", moves=np.array([k for k, _, _ in moves], np.int32),
               move_R=np.array([R for _, R, _ in moves]), move_t=np.array([t for _, _, t in moves]))
    for step in range(len(moves) + 1):
        if step:
            k, Rm, t = moves[step - 1]
            m.move_body(k, Rm, t)
        h = m.calculate()
        coords = np.concatenate([m.body_coords(b) for b in range(len(bodies))])
        aa, aw, ww_h = h.simple()
        tot, d = h.total()
        out[f"coords{step}"] = coords
        out[f"waters{step}"] = m.body_coords(-1)
        for key, v in (("aa", aa), ("aw", aw), ("ww", ww_h), ("tot", tot), ("d_axis", d)):
            out[f"{key}{step}"] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "steps", len(moves) + 1, "bins", len(out["d_axis0"]))


def hydrate_case(name, xyz, ff, body_sizes, noise_seed, moves=()):
    """Molecule::generate_new_hydration() (RadialHydration, no culling) with the noise table
    O.hydrate_noise(26 n, noise_seed + step) (one row per candidate; none when noise_seed is None), on
    a fresh grid; then after each rigid move (body, R, t) made as the rigid-body transforms make it
    (the body leaves the grid and is appended back, the axes are kept), again.  Per step: the grid's
    atoms in visiting order, the waters in body order, the waters per body and the grid axes."""
    O.ref_set_axes(0.25, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(False)
    m = O.RefMolecule(xyz, np.ones(len(xyz)), ff, np.zeros((0, 3)), np.zeros(0), body_sizes=list(body_sizes))
    out = dict(body_sizes=np.asarray(body_sizes, np.int32), manager="hydrate", steps=len(moves) + 1,
               moves=np.array([k for k, _, _ in moves], np.int32), noise_seed=-1 if noise_seed is None else noise_seed)
    for step in range(len(moves) + 1):
        if step:
            k, Rm, t = moves[step - 1]
            m.move_body_in_grid(k, Rm, t)
        noise = None if noise_seed is None else O.hydrate_noise(26 * len(xyz), noise_seed + step)
        a, w, per_body, axes, _ = m.hydrate(noise, fresh_grid=(step == 0), n_bodies=len(body_sizes))
        out[f"atoms{step}"] = a[:, :3].copy()
        out[f"ff{step}"] = a[:, 3].astype(np.int32)
        out[f"waters{step}"] = w
        out[f"per_body{step}"] = per_body
        out[f"axes{step}"] = np.concatenate([axes[:3], axes[6:]])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "waters", [len(out[f"waters{s}"]) for s in range(len(moves) + 1)])


def main():
    O.ref()
    # SimpleCube: 8 corners + centre as atoms (carbon), 8 corner waters
    atoms = np.vstack([CUBE, [[0, 0, 0]]])
    ff = np.full(9, 3)
    w = np.ones(9)
    waters = CUBE.copy()
    ww = np.ones(8)
    for mgr in ("mt", "ffavg", "ffexplicit"):
        run_case(f"cube_{mgr}", atoms, ff, w, waters, ww, np.zeros((0, 3)), 100.0, 0.25, mgr)
    run_case("cube_ffgrid", atoms, ff, w, waters, ww, CUBE * 2.0, 100.0, 0.25, "ffgrid")

    rng = np.random.default_rng(20240601)
    elements = np.array([3, 7, 11, 12])
    charge = {3: 5.997198, 7: 6.996361, 11: 7.999706, 12: 15.989624}
    for k, (na, nw, nx, bw) in enumerate([(257, 63, 0, 0.25), (401, 97, 0, 0.1), (130, 0, 0, 0.25),
                                          (333, 71, 250, 0.1)]):
        xyz = rng.normal(0, 7, (na, 3))
        f = rng.choice(elements, na, p=[0.63, 0.17, 0.19, 0.01])
        wt = np.array([charge[t] for t in f]) * rng.uniform(0.8, 1.2, na)
        wat = rng.normal(0, 9, (nw, 3))
        wwt = np.full(nw, 8.999659)
        exv = np.round(rng.uniform(-9, 9, (nx, 3)))
        vol = 40.0 * na
        run_case(f"random{k}_mt", xyz, f, wt, wat, wwt, exv, vol, bw, "mt", cw=1.3)
        run_case(f"random{k}_ffavg", xyz, f, wt, wat, wwt, exv, vol, bw, "ffavg", cw=1.1, cx=0.97, crho=1.02,
                 dwa=0.4, dwx=0.2)
        run_case(f"random{k}_ffexplicit", xyz, f, wt, wat, wwt, exv, vol, bw, "ffexplicit", cw=1.1, cx=0.97,
                 crho=1.02, dwa=0.4, dwx=0.2)
        if nx:
            run_case(f"random{k}_ffgrid", xyz, f, wt, wat, wwt, exv, vol, bw, "ffgrid", cw=0.9, cx=1.05)
    # Real proteins from the reference's own test files (tests/files in the reference), read by the
    # reference's reader, so the atoms carry its united-atom form-factor types (CH, CH2, NH, OH, ...)
    files = os.path.join(REF_ROOT, "tests", "files")
    for pdb in ("2epe", "6lyz"):
        path = os.path.join(files, pdb + ".pdb")
        if not os.path.exists(path):
            continue
        xyz, wt, f, wat, wwt = O.ref_read_structure(path)
        vol = 18.0 * len(xyz)
        run_case(f"pdb_{pdb}_mt", xyz, f, wt, wat, wwt, np.zeros((0, 3)), vol, 0.25, "mt", cw=1.2)
        run_case(f"pdb_{pdb}_ffavg", xyz, f, wt, wat, wwt, np.zeros((0, 3)), vol, 0.25, "ffavg", cw=1.05, cx=0.98,
                 crho=1.01, dwa=0.3, dwx=0.1)
        run_case(f"pdb_{pdb}_ffexplicit", xyz, f, wt, wat, wwt, np.zeros((0, 3)), vol, 0.1, "ffexplicit", cw=1.05,
                 cx=1.02)
    # Grid excluded-volume dummies (RawGridExv::create on the expanded grid) and the grid volume
    grid_case("gridexv_cube", np.vstack([CUBE, [[0, 0, 0]]]), np.full(9, 3), CUBE.copy())
    for k, (na, nw, spread) in enumerate([(300, 60, 8.0), (1500, 300, 14.0)]):
        xyz = rng.normal(0, spread, (na, 3)).astype(np.float32).astype(np.float64)
        f = rng.choice([1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14], na)
        wat = rng.normal(0, spread * 1.2, (nw, 3)).astype(np.float32).astype(np.float64)
        grid_case(f"gridexv_random{k}", xyz, f, wat)
    path = os.path.join(files, "2epe.pdb")
    if os.path.exists(path):
        xyz, _, f, wat, _ = O.ref_read_structure(path)
        grid_case("gridexv_2epe", xyz.astype(np.float32).astype(np.float64), f, wat.astype(np.float32).astype(np.float64))
    # SimpleCalculator job lists (seeded stream of their own)
    crng = np.random.default_rng(11)

    def pts(n, spread):
        return np.column_stack([crng.normal(0, spread, (n, 3)), crng.uniform(0.5, 8.0, n)]).astype(np.float32)

    sets = [pts(n, 7.0) for n in (257, 64, 131, 33)]
    calc_case("calc_random_merge", sets, [(0, None, 4, 0), (1, None, 1, 0), (0, 1, 3, 0), (2, 0, 1, 0), (0, 2, 2, 1),
                                          (3, None, 60, 1), (3, 1, 7, -1), (2, None, 1, -1), (1, 2, 5, 2)], 0.25)
    # a body with a 5-fold cyclic copy chain: self x 5, the chain's distinct pairs with their multiplicities
    body = pts(300, 5.0)
    ang = 2 * np.pi / 5
    rot = lambda k: np.array([[np.cos(k * ang), -np.sin(k * ang), 0], [np.sin(k * ang), np.cos(k * ang), 0], [0, 0, 1]])
    copies = [np.column_stack([(body[:, :3].astype(np.float64) + [14.0, 0, 0]) @ rot(k).T, body[:, 3]]).astype(np.float32)
              for k in range(5)]
    waters = pts(80, 16.0)
    calc_case("calc_cyclic5", copies + [waters], [(0, None, 5, 0), (0, 1, 5, 0), (0, 2, 5, 0)] +
              [(5, k, 1, 1) for k in range(5)] + [(5, None, 1, 2)], 0.1)
    # PartialHistogramManagerMT: four bodies, waters, two rigid moves (seeded stream of its own)
    prng = np.random.default_rng(13)
    bodies = [prng.normal(c, 4.0, (n, 3)) for c, n in (((0, 0, 0), 180), ((12, 0, 0), 120), ((0, 13, 2), 150),
                                                         ((-9, -8, 5), 90))]
    ws = [prng.uniform(4.0, 9.0, len(b)) for b in bodies]
    waters = prng.normal(0, 12, (70, 3))
    ww = np.full(70, 8.999659)
    moves = [(2, rotation((1, 2, 0.5), 0.07), np.array([0.8, -1.1, 0.4])),
             (0, rotation((0.2, -1, 1), 0.05), np.array([-0.5, 0.3, 1.2]))]
    partial_case("partial_random_4bodies", bodies, ws, waters, ww, moves, 0.25)
    # hydration shells (RadialHydration), seeded streams of their own
    hrng = np.random.default_rng(17)
    xyz = hrng.normal(0, 6, (300, 3))
    f = hrng.choice([2, 3, 4, 7, 8, 11, 12, 14], 300)
    hydrate_case("hydrate_random_2bodies", xyz, f, [180, 120], 171)
    xyz = hrng.normal(0, 10, (1500, 3))
    f = hrng.choice(elements, 1500)
    hydrate_case("hydrate_random_nonoise", xyz, f, [1500], None)
    xyz = np.concatenate([hrng.normal(c, 4.0, (n, 3)) for c, n in (((0, 0, 0), 200), ((14, 0, 0), 150), ((0, 15, 3), 120))])
    f = hrng.choice(elements, len(xyz))
    hydrate_case("hydrate_moves_3bodies", xyz, f, [200, 150, 120], 173,
                 moves=[(0, rotation((1, 0.3, -0.4), 0.3), np.array([-6.0, 2.0, 1.0])),
                        (2, rotation((0, 1, 0), -0.2), np.array([3.0, 9.0, -2.0]))])
    path = os.path.join(files, "2epe.pdb")
    if os.path.exists(path):
        xyz, _, f, _, _ = O.ref_read_structure(path)
        hydrate_case("hydrate_pdb_2epe", xyz, f, [len(xyz)], 175)
    # SmartFitter fits with the Golden minimiser, one parameter each (seeded noise streams of their own)
    frng = np.random.default_rng(7)
    xyz = frng.normal(0, 9, (400, 3))
    f = frng.choice(elements, 400, p=[0.63, 0.17, 0.19, 0.01])
    wt = np.array([charge[t] for t in f])
    wat = frng.normal(0, 11, (90, 3))
    wwt = np.full(90, 8.999659)
    exv = np.round(frng.uniform(-9, 9, (300, 3)))
    fit_case("fit_random_mt_cw", xyz, f, wt, wat, wwt, np.zeros((0, 3)), 18.0 * 400, 0.25, "mt", 0, 1.4, 101)
    fit_case("fit_random_ffavg_cw", xyz, f, wt, wat, wwt, np.zeros((0, 3)), 18.0 * 400, 0.25, "ffavg", 0, 1.6, 102)
    fit_case("fit_random_ffavg_dwa", xyz, f, wt, wat, wwt, np.zeros((0, 3)), 18.0 * 400, 0.25, "ffavg", 3, 0.7, 103)
    fit_case("fit_random_ffgrid_cx", xyz, f, wt, wat, wwt, exv, 18.0 * 400, 0.1, "ffgrid", 1, 1.03, 104)
    fit_case("fit_random_ffexplicit_crho", xyz, f, wt, wat, wwt, np.zeros((0, 3)), 18.0 * 400, 0.1, "ffexplicit", 2,
             1.15, 105)
    path = os.path.join(files, "2epe.pdb")
    if os.path.exists(path):
        xyz, wt, f, wat, wwt = O.ref_read_structure(path)
        fit_case("fit_pdb_2epe_ffavg_cw", xyz, f, wt, wat, wwt, np.zeros((0, 3)), 18.0 * len(xyz), 0.25, "ffavg", 0,
                 2.2, 106)
    # Simple excluded volume enabled (weights shifted by -rho_w V / N, SimpleExvModel.cpp:23-28)
    xyz = rng.normal(0, 6, (120, 3))
    f = rng.choice(elements, 120)
    wt = np.array([charge[t] for t in f])
    run_case("random_simple_exv_mt", xyz, f, wt, np.zeros((0, 3)), np.zeros(0), np.zeros((0, 3)), 900.0, 0.25, "mt",
             simple_exv=True)


def reference_hist(m, manager, bin_width, q):
    """The reference's histograms of a molecule and the oracle's I(q) of them at q."""
    import time

    O.ref_set_axes(bin_width, 8000, 1e-4, 1.0)
    O.ref_set_simple_exv(False)
    rm = O.RefMolecule(m.atoms, m.weights, m.ff_types, m.waters, m.water_weights, volume=m.volume)
    rm.set_manager(manager, exv_xyz=m.exv if manager == "ffgrid" else None)
    t0 = time.perf_counter()
    h = rm.calculate()
    secs = time.perf_counter() - t0
    aa, aw, ww = h.ff()
    tot, d = h.total()
    # raw doubles: pair counts, and for FFAvg the excluded-volume rows scaled by Z_exv
    out = dict(aa=aa, aw=aw, ww_h=ww, tot=tot, d_axis=d)
    kind = {"ffavg": 0, "ffgrid": 2}[manager]
    ax = xx = None
    if manager == "ffgrid":
        ax, xx = h.grid_axes()
        ax, xx = ax[: len(d)], xx[: len(d)]
        out["d_axis_ax"], out["d_axis_xx"] = ax, xx
    fh = O.FFHist(aa, aw, ww, tot, d, ax, xx)
    out["q"] = np.asarray(q, np.float64)
    out["Iq"], _ = O.debye_ff(kind, fh, out["q"])
    return out, secs


def fullsize():
    from ausaxs_b200 import synth

    O.ref()
    which = sys.argv[2:] or ["cfg1", "cfg2", "cfg3"]
    for name, wl in (("fullsize_cfg1", synth.cfg1() if "cfg1" in which else None),
                     ("fullsize_cfg2", synth.cfg2() if "cfg2" in which else None)):
        if wl is None:
            continue
        m = wl.molecules[0]
        out, secs = reference_hist(m, wl.manager, wl.bin_width, wl.q)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), digest=input_digest(m), workload=wl.name,
                            manager=wl.manager, bin_width=wl.bin_width, **out)
        print(name, "bins", len(out["d_axis"]), f"{secs:.1f} s")
    if "cfg3" not in which:
        return
    wl = synth.cfg3()
    ranked = sorted(range(len(wl.molecules)), key=lambda i: -wl.molecules[i].size_atom())
    picks = [ranked[int(round(k * (len(ranked) - 1) / 7))] for k in range(8)]
    store = {"indices": np.array(picks, np.int64), "workload": wl.name, "manager": wl.manager,
             "bin_width": wl.bin_width}
    for k, i in enumerate(picks):
        m = wl.molecules[i]
        out, secs = reference_hist(m, wl.manager, wl.bin_width, wl.q)
        store[f"digest{k}"] = input_digest(m)
        for key, v in out.items():
            store[f"{key}{k}"] = v
        print("cfg3 structure", i, m.size_atom(), "atoms", f"{secs:.1f} s")
    np.savez_compressed(os.path.join(HERE, "fullsize_cfg3.npz"), **store)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "fullsize":
        fullsize()
    else:
        main()
