"""Seeded synthetic workloads (the benchmark configurations and the test structures).

No public dataset is involved: every structure is generated from a seed by ``csrc/synth.c``
(random-walk globules, hydration shells, grid excluded-volume dummies) and assembled here.

Workloads (sizes as the benchmark configurations state them):
  cfg0  5,000-atom globule (Rg ~18 A), 1,000 shell waters, 0.25 A bins, 200 q in [0.005, 0.5]
  cfg1  50,000-atom globule (Rg ~40 A), 10,000 waters, 1 A grid excluded volume, 0.1 A bins,
        1,000 q in [0.005, 1.0]
  cfg2  60 icosahedral copies of an 8,333-atom subunit in a 120-150 A shell, 60,000 waters,
        0.1 A bins, 2,000 q in [0.005, 1.0]
  cfg3  256 globules, N log-uniform in [500, 50,000], waters 20 % of N, 0.25 A bins,
        400 q in [0.005, 0.8]
  cfg4  64 chains of 8-body assemblies (3,000-20,000 atoms per body), 400 q in [0.005, 0.5]
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .hist import Molecule

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

ELEMENT_FRACTIONS = (0.63, 0.17, 0.19, 0.01)  # C, N, O, S
FF_C, FF_N, FF_O, FF_S, FF_WATER = 3, 7, 11, 12, 1


def _synth():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_lib", "libsynth.so")
        if not os.path.exists(path):
            from .build import build_synth

            build_synth()
        L = C.CDLL(path)
        f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.synth_globule.restype = C.c_int
        L.synth_globule.argtypes = [C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_double, f64, f64, i32]
        L.synth_waters.restype = C.c_int
        L.synth_waters.argtypes = [C.c_uint64, f64, i32, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, f64]
        L.synth_exv_grid.restype = C.c_int
        L.synth_exv_grid.argtypes = [f64, i32, C.c_int, C.c_double, C.c_void_p, C.c_int]
        _lib = L
    return _lib


def ff_charge(ff: np.ndarray) -> np.ndarray:
    """Effective charge of a form-factor type: the five-Gaussian form factor at q = 0
    (constants::charge::get_ff_charge), for the Simple (weights) model."""
    table = {1: 8.999659, 3: 5.997198, 7: 6.996361, 11: 7.999706, 12: 15.989624}
    return np.array([table[int(t)] for t in ff], np.float64)


def globule(seed: int, n: int, rg: float = None, r_in: float = 0.0, r_out: float = None, cone_cos: float = -2.0):
    """Self-avoiding random walk of n atoms; returns (xyz [n,3], ff [n])."""
    if r_out is None:
        rg = rg if rg is not None else 18.0 * (n / 5000.0) ** (1.0 / 3.0)
        r_out = rg / np.sqrt(3.0 / 5.0)
    xyz = np.zeros(3 * n)
    ff = np.zeros(n, np.int32)
    frac = np.cumsum(ELEMENT_FRACTIONS).astype(np.float64)
    got = _synth().synth_globule(seed, n, r_in, r_out, cone_cos, frac, xyz, ff)
    if got != n:
        raise RuntimeError(f"globule generator placed {got} of {n} atoms")
    return xyz.reshape(n, 3), ff


def waters(seed: int, xyz: np.ndarray, ff: np.ndarray, n: int, shell=(2.5, 3.5), min_sep: float = 0.0) -> np.ndarray:
    if n == 0:
        return np.zeros((0, 3))
    out = np.zeros(3 * n)
    got = _synth().synth_waters(seed, np.ascontiguousarray(xyz.reshape(-1)), np.ascontiguousarray(ff), len(ff), n,
                                shell[0], shell[1], min_sep, out)
    return out[: 3 * got].reshape(got, 3)


def exv_grid(xyz: np.ndarray, ff: np.ndarray, width: float = 1.0) -> np.ndarray:
    L = _synth()
    x = np.ascontiguousarray(xyz.reshape(-1))
    f = np.ascontiguousarray(ff)
    m = L.synth_exv_grid(x, f, len(ff), width, None, 0)
    out = np.zeros(3 * m)
    L.synth_exv_grid(x, f, len(ff), width, out.ctypes.data, m)
    return out.reshape(m, 3)


def icosahedral_rotations() -> np.ndarray:
    """The 60 proper rotations of the icosahedral group, by closure of a 5-fold and a 3-fold generator."""
    phi = (1 + 5 ** 0.5) / 2

    def rot(axis, ang):
        a = np.asarray(axis, float)
        a /= np.linalg.norm(a)
        K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
        return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K

    gens = [rot([0, 1, phi], 2 * np.pi / 5), rot([1, 1, 1], 2 * np.pi / 3)]
    group = [np.eye(3)]
    frontier = [np.eye(3)]
    while frontier:
        new = []
        for g in frontier:
            for h in gens:
                m = h @ g
                if not any(np.allclose(m, x, atol=1e-9) for x in group):
                    group.append(m)
                    new.append(m)
        frontier = new
    assert len(group) == 60
    return np.array(group)


def random_rotation(rng: np.random.Generator, max_deg: float) -> np.ndarray:
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    ang = np.deg2rad(rng.uniform(0, max_deg))
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K


@dataclass
class Workload:
    name: str
    molecules: List[Molecule]
    bin_width: float
    q: np.ndarray
    manager: str
    bin_count: int = 8000
    extra: dict = field(default_factory=dict)


def _molecule(seed, n, n_w, rg=None, exv_width=None, volume_from_grid=True):
    xyz, ff = globule(seed, n, rg)
    w = waters(seed + 1, xyz, ff, n_w)
    exv = exv_grid(xyz, ff, exv_width or 1.0)
    vol = float(len(exv)) * (exv_width or 1.0) ** 3
    return Molecule(atoms=xyz, ff_types=ff, weights=ff_charge(ff), waters=w,
                    water_weights=np.full(len(w), ff_charge([FF_WATER])[0]),
                    exv=exv if exv_width else None, volume=vol)


def cfg0(seed: int = 1) -> Workload:
    m = _molecule(seed, 5000, 1000, rg=18.0)
    return Workload("cfg0: 5k-atom globule + 1k waters, FFAvg, 0.25 A bins, 200 q", [m], 0.25,
                    np.linspace(0.005, 0.5, 200), "ffavg")


def cfg1(seed: int = 11, atoms: int = 50000) -> Workload:
    """atoms != 50000: the same composition and density (Rg ~ atoms^(1/3), waters atoms/5), for
    profiling cases of the same kernels."""
    rg = 40.0 * (atoms / 50000) ** (1.0 / 3.0)
    m = _molecule(seed, atoms, atoms // 5, rg=rg, exv_width=1.0)
    name = "cfg1: 50k atoms + 10k waters" if atoms == 50000 else f"cfg1 shape: {atoms} atoms + {atoms // 5} waters"
    return Workload(name + " + 1 A grid exv, FFGrid, 0.1 A bins, 1000 q", [m], 0.1, np.linspace(0.005, 1.0, 1000),
                    "ffgrid")


def cfg2(seed: int = 21, subunit: int = 8333) -> Workload:
    cos_half = 1.0 - 1.0 / 36.0
    sub, ff = globule(seed, subunit, r_in=120.0, r_out=150.0, cone_cos=cos_half)
    R = icosahedral_rotations()
    xyz = np.concatenate([sub @ r.T for r in R])
    ffs = np.tile(ff, len(R))
    w = waters(seed + 1, xyz, ffs, 60000)
    m = Molecule(atoms=xyz, ff_types=ffs, weights=ff_charge(ffs), waters=w,
                 water_weights=np.full(len(w), ff_charge([FF_WATER])[0]), volume=float(len(xyz)) * 11.0)
    name = "cfg2: 500k-atom icosahedral shell" if subunit == 8333 else f"cfg2 shape: {len(xyz)}-atom icosahedral shell"
    return Workload(name + " + 60k waters, FFAvg, 0.1 A bins, 2000 q", [m], 0.1, np.linspace(0.005, 1.0, 2000), "ffavg")


def _molecule_args(args):
    return _molecule(*args)


def cfg3(seed: int = 31, count: int = 256, nmin: int = 500, nmax: int = 50000) -> Workload:
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(int)
    jobs = [(seed * 1000 + i, int(n), int(round(0.2 * n))) for i, n in enumerate(ns)]
    workers = min(16, os.cpu_count() or 1)
    if count >= 16 and workers > 1:
        # spawn: safe after CUDA has been initialised in the parent
        import concurrent.futures
        import multiprocessing
        with concurrent.futures.ProcessPoolExecutor(workers, mp_context=multiprocessing.get_context("spawn")) as ex:
            mols = list(ex.map(_molecule_args, jobs, chunksize=4))
    else:
        mols = [_molecule(*j) for j in jobs]
    return Workload(f"cfg3: {count} globules, N log-uniform [{nmin}, {nmax}], FFAvg, 0.25 A bins, 400 q", mols, 0.25,
                    np.linspace(0.005, 0.8, 400), "ffavg")


@dataclass
class Assembly:
    """A multi-body assembly for the rigid-body serving workload."""

    bodies: List[np.ndarray]      # per body [n, 3]
    ff: List[np.ndarray]
    weights: List[np.ndarray]


def assembly(seed: int, n_bodies: int = 8, nmin: int = 3000, nmax: int = 20000) -> Assembly:
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_bodies)).astype(int)
    bodies, ffs, ws = [], [], []
    radii = [18.0 * (n / 5000.0) ** (1 / 3) / np.sqrt(0.6) for n in ns]
    spacing = 2 * max(radii) + 4.0
    side = int(np.ceil(n_bodies ** (1 / 3)))
    for b, n in enumerate(ns):
        xyz, ff = globule(seed * 100 + b, int(n))
        ix, iy, iz = b % side, (b // side) % side, b // (side * side)
        xyz = xyz + np.array([ix, iy, iz], float) * spacing
        bodies.append(xyz)
        ffs.append(ff)
        ws.append(ff_charge(ff))
    return Assembly(bodies, ffs, ws)


def radius_of_gyration(xyz: np.ndarray) -> float:
    c = xyz.mean(axis=0)
    return float(np.sqrt(((xyz - c) ** 2).sum(axis=1).mean()))
