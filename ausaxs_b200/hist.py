"""Host-side mirror of the reference's histogram-manager and composite-histogram interfaces.

Names, arguments and results follow the reference so that code written against
``hist::IHistogramManager`` / ``ICompositeDistanceHistogram(Exv)`` reads the same:

* ``HistogramManagerMT`` / ``HistogramManagerMTFFAvg`` / ``HistogramManagerMTFFExplicit`` /
  ``HistogramManagerMTFFGrid`` -- ``calculate_all()`` as in
  source/core/hist/histogram_manager/HistogramManager{MT,MTFFAvg,MTFFExplicit,MTFFGrid}.cpp;
* ``CompositeDistanceHistogram`` (Simple, source/core/hist/intensity_calculator/CompositeDistanceHistogram.cpp)
  and ``CompositeDistanceHistogramFFAvg`` / ``...FFGrid`` (CompositeDistanceHistogramFFAvgBase.cpp,
  CompositeDistanceHistogramFFGrid.cpp) with ``apply_*_factor``, ``debye_transform`` and
  ``get_profile_*``.

All computation runs in the CUDA library through the C ABI (include/ausaxs_b200.h); this module
only marshals arrays.  Settings the reference reads from globals (bin width/count, weighted bins,
q range) are explicit arguments here.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _capi
from ._capi import AusaxsError, DebyeParams, HistConfig, HistResult, check, dptr, fptr, load

NFF = 15
RHO_WATER = 0.334  # e/A^3, constants::charge::density::water (include/core/constants/Constants.h:114)


def default_q_axis(qmin: float = 1e-4, qmax: float = 0.5) -> np.ndarray:
    """constants::axes::q_axis = Axis(1e-4, 1, 200) restricted by sub_axis(qmin, qmax)
    (include/core/constants/ConstantsAxes.h:14, source/core/utility/Axis.cpp:40-59)."""
    lo, hi, bins = 1e-4, 1.0, 200
    w = (hi - lo) / bins

    def get_bin(v):
        if v <= lo:
            return 0
        if v >= hi:
            return bins
        return int(np.floor((v + 1e-6 - lo) / w))

    b0, b1 = get_bin(qmin), get_bin(qmax)
    new_min, new_max = lo + b0 * w, lo + b1 * w
    n = b1 - b0
    ww = (new_max - new_min) / n
    return np.array([new_min + i * ww for i in range(n)])


def pack(xyz, fourth, as_int: bool) -> np.ndarray:
    """float32 [n, 4] compact records {x, y, z, w | ff} (CompactCoordinatesXYZW.h:131-134)."""
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    out = np.empty((len(xyz), 4), np.float32)
    out[:, :3] = xyz.astype(np.float32)
    if as_int:
        out[:, 3] = np.asarray(fourth, np.int32).reshape(-1).view(np.float32)
    else:
        out[:, 3] = np.asarray(fourth, np.float64).reshape(-1).astype(np.float32)
    return np.ascontiguousarray(out)


# constants::charge::get_ff_charge(WATER): the weight data::Water carries (Water.h:15-18)
WATER_CHARGE = 8.999659


@dataclass
class Molecule:
    """The inputs of the hot path a data::Molecule provides: atoms with form-factor type and
    weight, hydration waters, optional grid excluded-volume dummies, and the molecular volume
    used for the average excluded-volume charge (Molecule::get_volume_grid)."""

    atoms: np.ndarray                       # [n, 3] coordinates
    ff_types: Optional[np.ndarray] = None   # [n] form_factor_t
    weights: Optional[np.ndarray] = None    # [n] effective charges
    waters: Optional[np.ndarray] = None     # [m, 3]
    water_weights: Optional[np.ndarray] = None
    exv: Optional[np.ndarray] = None        # [k, 3] grid dummies (FFGrid); None: from the molecular grid
    volume: Optional[float] = None          # None: the molecular grid's volume (Molecule::get_volume_grid)

    def size_atom(self) -> int:
        return len(self.atoms)

    def size_water(self) -> int:
        return 0 if self.waters is None else len(self.waters)

    def get_volume_grid(self) -> float:
        """The given volume, or the volume of the molecular grid computed on the device
        (Molecule::get_volume_grid, source/core/data/Molecule.cpp:147-150)."""
        if self.volume is not None:
            return float(self.volume)
        a, w, _ = self.compact_ff()
        return _capi.grid_exv(_capi.default_context(), a, w)[1]

    def generate_new_hydration(self, noise=None, seed: int = 0, ctx: Optional[_capi.Context] = None) -> int:
        """Molecule::generate_new_hydration() (source/core/data/Molecule.cpp:219-226) with the reference's
        default RadialHydration and no culling, on the device: replaces the waters (weighted by the
        water form factor's charge, as data::Water is) and returns their count.  noise: one
        displacement per candidate ([n * 26, 3]), else seed != 0 draws Gaussian ones (sigma 0.75 A)
        on the device, else none."""
        w, _, _ = _capi.hydrate(ctx or _capi.default_context(), self.atoms, self.ff_types, None, noise, seed)
        self.waters = w
        self.water_weights = np.full(len(w), WATER_CHARGE)
        return len(w)

    def compact_ff(self):
        a = pack(self.atoms, self.ff_types, True)
        w = pack(self.waters if self.waters is not None else np.zeros((0, 3)), np.ones(self.size_water(), np.int32), True)
        x = pack(self.exv if self.exv is not None else np.zeros((0, 3)), np.zeros(0 if self.exv is None else len(self.exv), np.int32), True)
        return a, w, x

    def compact_w(self):
        a = pack(self.atoms, self.weights, False)
        ww = self.water_weights if self.water_weights is not None else np.zeros(self.size_water())
        w = pack(self.waters if self.waters is not None else np.zeros((0, 3)), ww, False)
        return a, w


class _Composite:
    """Common part of the composite histograms returned by the managers."""

    kind = 0

    def __init__(self, cfg: HistConfig, res: dict, ctx):
        self._cfg = cfg
        self._r = res
        self._ctx = ctx
        self.max_bin = int(res["max_bin"])
        self.pairs = int(res["pairs"])
        self.free = dict(cw=1.0, cx=1.0, crho=1.0, dw_atomic=0.0, dw_exv=0.0)
        self.grid_width = 1.0
        # 0: split-BF16 tensor cores + FP64 for the q whose error estimate exceeds `tolerance`;
        # 1: FP64 for every q
        self.precision = 1
        self.tolerance = 1e-5

    # DistanceHistogram interface
    def get_d_axis(self) -> np.ndarray:
        return self._r["d_axis"]

    def get_counts(self) -> np.ndarray:
        return self._r["tot"]

    def apply_water_scaling_factor(self, k: float):
        self.free["cw"] = float(k)

    def _result(self) -> HistResult:
        r = HistResult()
        r.max_bin = self.max_bin
        self._keep = {k: np.ascontiguousarray(v) for k, v in self._r.items() if isinstance(v, np.ndarray)}
        for name in ("aa", "aw", "ww", "tot", "d_axis", "d_axis_ax", "d_axis_xx"):
            setattr(r, name, dptr(self._keep.get(name)))
        return r

    def _transform(self, q):
        q = default_q_axis() if q is None else np.ascontiguousarray(q, np.float64)
        p = DebyeParams(self.free["cw"], self.free["cx"], self.free["crho"], self.free["dw_atomic"],
                        self.free["dw_exv"], self.grid_width, self.precision, self.tolerance)
        I = np.zeros(len(q))
        prof = np.zeros(6 * len(q))
        r = self._result()
        check(load().ausaxs_gpu_debye(self._ctx.h, C.byref(self._cfg), C.byref(r), dptr(q), len(q), C.byref(p),
                                      dptr(I), dptr(prof)))
        return q, I, prof.reshape(6, len(q))

    def debye_transform(self, q: Optional[Sequence[float]] = None):
        """I(q) at q (default: the reference's default q axis within [qmin, qmax])."""
        q, I, _ = self._transform(q)
        return q, I

    def profiles(self, q=None) -> np.ndarray:
        """[6][nq] partial profiles {aa, ax, aw, xx, wx, ww}."""
        return self._transform(q)[2]

    def get_profile_aa(self, q=None):
        return self.profiles(q)[0]

    def get_profile_aw(self, q=None):
        return self.profiles(q)[2]

    def get_profile_ww(self, q=None):
        return self.profiles(q)[5]


class CompositeDistanceHistogram(_Composite):
    """Simple (weights) composite histogram: aa, aw, ww weighted counts."""

    def get_aa_counts(self):
        return self._r["aa"]

    def get_aw_counts(self):
        return self._r["aw"]

    def get_ww_counts(self):
        return self._r["ww"]


class CompositeDistanceHistogramFFAvg(_Composite):
    def get_raw_aa_counts_by_ff(self):
        return self._r["aa"]

    def get_raw_aw_counts_by_ff(self):
        return self._r["aw"]

    def get_raw_ww_counts_by_ff(self):
        return self._r["ww"]

    def apply_excluded_volume_scaling_factor(self, k: float):
        self.free["cx"] = float(k)

    def apply_solvent_density_scaling_factor(self, k: float):
        self.free["crho"] = float(k)

    def apply_atomic_debye_waller_factor(self, s: float):
        self.free["dw_atomic"] = float(s)

    def apply_exv_debye_waller_factor(self, s: float):
        self.free["dw_exv"] = float(s)

    def get_profile_ax(self, q=None):
        return self.profiles(q)[1]

    def get_profile_xx(self, q=None):
        return self.profiles(q)[3]

    def get_profile_wx(self, q=None):
        return self.profiles(q)[4]


class CompositeDistanceHistogramFFExplicit(CompositeDistanceHistogramFFAvg):
    pass


class CompositeDistanceHistogramFFGrid(CompositeDistanceHistogramFFAvg):
    def get_d_axis_ax(self):
        return self._r["d_axis_ax"]

    def get_d_axis_xx(self):
        return self._r["d_axis_xx"]


class _Manager:
    manager = 0
    composite = _Composite

    def __init__(self, protein: Molecule, weighted_bins: bool = True, bin_width: float = 0.25, bin_count: int = 8000,
                 ctx: Optional[_capi.Context] = None):
        self.protein = protein
        self.weighted_bins = weighted_bins
        self.bin_width = bin_width
        self.bin_count = bin_count
        self.ctx = ctx or _capi.default_context()

    def config(self) -> HistConfig:
        z = 0.0
        if self.manager == _capi.MANAGER_FFAVG and self.protein.size_atom():
            # without a given volume the device takes Z_exv from the molecular grid (z_exv < 0)
            z = -1.0 if self.protein.volume is None else self.protein.get_volume_grid() * RHO_WATER / self.protein.size_atom()
        return HistConfig(self.manager, int(self.weighted_bins), float(self.bin_width), int(self.bin_count), z)

    def _inputs(self):
        raise NotImplementedError

    def _exv_count(self, x) -> int:
        if x is not None:
            return len(x)
        return _capi.EXV_FROM_GRID if self.manager == _capi.MANAGER_FFGRID else 0

    def calculate_all(self):
        cfg = self.config()
        a, w, x = self._inputs()
        nb = self.bin_count
        ff = self.manager != _capi.MANAGER_MT
        bufs = {
            "aa": np.zeros(NFF * NFF * nb if ff else nb),
            "aw": np.zeros(NFF * nb if ff else nb),
            "ww": np.zeros(nb),
            "tot": np.zeros(nb),
            "d_axis": np.zeros(nb),
            "d_axis_ax": np.zeros(nb),
            "d_axis_xx": np.zeros(nb),
        }
        r = HistResult()
        for k, v in bufs.items():
            setattr(r, k, dptr(v))
        check(load().ausaxs_gpu_histogram(self.ctx.h, C.byref(cfg), fptr(a), len(a), fptr(w), len(w), fptr(x),
                                          self._exv_count(x), C.byref(r)))
        m = r.max_bin
        res = {"max_bin": m, "pairs": r.pairs}
        if ff:
            res["aa"] = bufs["aa"][: NFF * NFF * m].reshape(NFF, NFF, m).copy()
            res["aw"] = bufs["aw"][: NFF * m].reshape(NFF, m).copy()
        else:
            res["aa"] = bufs["aa"][:m].copy()
            res["aw"] = bufs["aw"][:m].copy()
        for k in ("ww", "tot", "d_axis"):
            res[k] = bufs[k][:m].copy()
        if self.manager == _capi.MANAGER_FFGRID:
            res["d_axis_ax"] = bufs["d_axis_ax"][:m].copy()
            res["d_axis_xx"] = bufs["d_axis_xx"][:m].copy()
        return self.composite(cfg, res, self.ctx)

    def calculate(self):
        return self.calculate_all()


class HistogramManagerMT(_Manager):
    """Weights (Simple excluded volume); HistogramManagerMT.cpp:23-75."""

    manager = _capi.MANAGER_MT
    composite = CompositeDistanceHistogram

    def _inputs(self):
        a, w = self.protein.compact_w()
        return a, w, None


class HistogramManagerMTFFAvg(_Manager):
    """Form factors with the average excluded volume; HistogramManagerMTFFAvg.cpp:194-372."""

    manager = _capi.MANAGER_FFAVG
    composite = CompositeDistanceHistogramFFAvg

    def _inputs(self):
        a, w, _ = self.protein.compact_ff()
        return a, w, None


class HistogramManagerMTFFExplicit(_Manager):
    """Form factors, no excluded-volume rows; HistogramManagerMTFFExplicit.cpp:216-437."""

    manager = _capi.MANAGER_FFEXPLICIT
    composite = CompositeDistanceHistogramFFExplicit

    def _inputs(self):
        a, w, _ = self.protein.compact_ff()
        return a, w, None


class HistogramManagerMTFFGrid(_Manager):
    """Form factors with grid excluded-volume dummies; HistogramManagerMTFFGrid.cpp:43-234.
    The dummies (RawGridExv::create in the reference) come from Molecule.exv."""

    manager = _capi.MANAGER_FFGRID
    composite = CompositeDistanceHistogramFFGrid

    def __init__(self, protein: Molecule, bin_width: float = 0.25, bin_count: int = 8000, ctx=None):
        super().__init__(protein, True, bin_width, bin_count, ctx)

    def _inputs(self):
        a, w, x = self.protein.compact_ff()
        return a, w, (x if self.protein.exv is not None else None)  # None: dummies from the molecular grid


def profile(manager: _Manager, q, cw=1.0, cx=1.0, crho=1.0, dw_atomic=0.0, dw_exv=0.0, grid_width=1.0,
            precision: int = 1, with_profiles: bool = False, tolerance: float = 1e-5):
    """Coordinates -> I(q) in one call (Molecule::get_histogram()->debye_transform()): only I(q) leaves the device."""
    cfg = manager.config()
    a, w, x = manager._inputs()
    q = np.ascontiguousarray(q, np.float64)
    I = np.zeros(len(q))
    prof = np.zeros(6 * len(q)) if with_profiles else None
    p = DebyeParams(cw, cx, crho, dw_atomic, dw_exv, grid_width, precision, tolerance)
    check(load().ausaxs_gpu_profile(manager.ctx.h, C.byref(cfg), fptr(a), len(a), fptr(w), len(w), fptr(x),
                                    manager._exv_count(x), dptr(q), len(q), C.byref(p), dptr(I), dptr(prof)))
    return (I, prof.reshape(6, len(q))) if with_profiles else I


def combine_partials(self_aa, cross_aa, aw, ww, bin_width: float) -> dict:
    """PartialHistogramManagerMT::calculate / calculate_all (PartialHistogramManagerMT.cpp:152-252): the
    master is the sum of every partial (its base is zero), p_tot = master truncated to max_bin (last
    non-zero value, at least 10), aa = self + cross partials, aw = water partials, ww, and the weighted
    axis of the master (WeightedDistribution1D.cpp:51-58, bin 0 pinned to 0).  Each partial is a
    (value, count, distance sum) triple of equal-length arrays."""
    parts = list(self_aa) + list(cross_aa) + list(aw) + ([ww] if ww is not None else [])
    n = len(parts[0][0])
    value, count, dsum = (np.zeros(n) for _ in range(3))
    for v, c, d in parts:
        value += v
        count += c
        dsum += d
    nz = np.nonzero(value[10:])[0]
    mb = int(nz[-1]) + 11 if len(nz) else 10
    aa = sum(v for v, _, _ in list(self_aa) + list(cross_aa))
    aw_v = sum((v for v, _, _ in aw), np.zeros(n))
    ww_v = ww[0] if ww is not None else np.zeros(n)
    width = (mb * bin_width) / mb  # Axis(0, mb * width, mb).width()
    cnt = count[:mb].astype(np.uint64).astype(np.uint32).astype(np.float64)
    bc = dsum[:mb]
    d_axis = ((bc == 0) * (np.arange(mb) * width) + bc) / ((cnt == 0) + cnt)
    d_axis[0] = 0.0
    return {"aa": aa[:mb].copy(), "aw": aw_v[:mb].copy(), "ww": ww_v[:mb].copy(), "tot": value[:mb].copy(),
            "d_axis": d_axis, "max_bin": mb}


class PartialHistogramManagerMT:
    """PartialHistogramManagerMT (source/core/hist/histogram_manager/PartialHistogramManagerMT.cpp:42-252)
    over the device SimpleCalculator: the partial histograms of every body (self), every pair of bodies
    (cross) and every body with the waters are kept; calculate_all() recomputes only those of bodies
    whose coordinates changed since the last call (a rigid move leaves a body's self partial as it was,
    as the reference does) and returns the composite of their sum.  The waters are the hydration of
    body `water_owner` and move with it (Body::rotate / Body::translate, Body.cpp:135-156, which then
    signal a modified hydration: the water self partial and every body-water partial are recomputed).
    bodies: [(xyz [n, 3], weights [n])]; waters: (xyz [m, 3], weights [m]) or None."""

    def __init__(self, bodies, waters=None, bin_width: float = 0.25, bin_count: int = 8000,
                 ctx: Optional[_capi.Context] = None, water_owner: int = 0):
        self.ctx = ctx or _capi.default_context()
        self.bin_width, self.bin_count = bin_width, bin_count
        self.xyz = [np.array(x, np.float64).reshape(-1, 3) for x, _ in bodies]
        self.records = [pack(x, w, False) for x, w in bodies]
        self.water_owner = water_owner
        self.water_xyz = None
        self.waters = None
        if waters is not None and len(waters[0]):
            self.water_xyz = np.array(waters[0], np.float64).reshape(-1, 3)
            self.waters = pack(self.water_xyz, waters[1], False)
        B = len(self.records)
        self.moved = [True] * B          # externally modified (initially every partial is computed)
        self.internal = [True] * B       # internally modified: the self partial is recomputed
        self.water_changed = self.waters is not None
        self.self_p, self.aw_p = [None] * B, [None] * B
        self.cross_p = {}
        self.ww_p = None

    def set_body_coordinates(self, k: int, xyz, internal: bool = False):
        """New coordinates of body k (a rigid move unless `internal`, which also recomputes its self partial)."""
        self.xyz[k] = np.array(xyz, np.float64).reshape(-1, 3)
        self.records[k] = pack(self.xyz[k], self.records[k][:, 3].copy(), False)
        self.moved[k] = True
        self.internal[k] = self.internal[k] or internal

    def set_water_coordinates(self, xyz):
        """New coordinates of the waters (a modified hydration)."""
        self.water_xyz = np.array(xyz, np.float64).reshape(-1, 3)
        self.waters = pack(self.water_xyz, self.waters[:, 3].copy(), False)
        self.water_changed = True

    def set_waters(self, xyz, weights):
        """A new hydration of any size (Molecule::generate_new_hydration after a move, SimpleController.cpp:76):
        the hydration counts as modified, so the water self partial and every body-water partial are
        recomputed (PartialHistogramManagerMT.cpp:82-108)."""
        xyz = np.array(xyz, np.float64).reshape(-1, 3)
        B = len(self.records)
        if len(xyz) == 0:
            self.water_xyz = self.waters = None
            self.ww_p, self.aw_p = None, [None] * B
        else:
            self.water_xyz = xyz
            self.waters = pack(xyz, np.asarray(weights, np.float64).reshape(-1), False)
        self.water_changed = True

    @staticmethod
    def _rigid(xyz, R, t):
        # Body::rotate then Body::translate: x <- R x (row sums left to right, Vector3.h:169-181), then x + t
        R = np.asarray(R, np.float64).reshape(3, 3)
        t = np.asarray(t, np.float64).reshape(3)
        x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
        rot = np.column_stack([R[i, 0] * x + R[i, 1] * y + R[i, 2] * z for i in range(3)])
        return rot + t

    def move_body(self, k: int, R, t):
        """Rigid move x <- R x + t of body k, and of the waters when body k holds them."""
        self.set_body_coordinates(k, self._rigid(self.xyz[k], R, t))
        if self.waters is not None and k == self.water_owner:
            self.set_water_coordinates(self._rigid(self.water_xyz, R, t))

    def calculate_all(self) -> "CompositeDistanceHistogram":
        B = len(self.records)
        calc = _capi.Calculator(self.ctx, self.bin_width, self.bin_count)
        jobs = []  # (kind, key) in enqueue order; merge ids: self k, cross i*B+j, water B*B+k, ww B*B+B
        for k in range(B):
            if self.internal[k]:
                calc.enqueue_calculate_self(self.records[k], 1, k)
                jobs.append(("self", k))
        if self.waters is not None and self.water_changed:
            calc.enqueue_calculate_self(self.waters, 1, B * B + B)
            jobs.append(("ww", None))
        for i in range(B):
            for j in range(i):
                if self.moved[i] or self.moved[j]:
                    calc.enqueue_calculate_cross(self.records[i], self.records[j], 1, i * B + j)
                    jobs.append(("cross", (i, j)))
            if self.waters is not None and (self.moved[i] or self.water_changed):
                calc.enqueue_calculate_cross(self.records[i], self.waters, 1, B * B + i)
                jobs.append(("aw", i))
        res = calc.run()
        calc.close()
        for kind, key in jobs:
            if kind == "self":
                self.self_p[key] = res["self"][key]
            elif kind == "ww":
                self.ww_p = res["self"][B * B + B]
            elif kind == "cross":
                self.cross_p[key] = res["cross"][key[0] * B + key[1]]
            else:
                self.aw_p[key] = res["cross"][B * B + key]
        self.moved = [False] * B
        self.internal = [False] * B
        self.water_changed = False
        r = combine_partials(self.self_p, list(self.cross_p.values()), [p for p in self.aw_p if p is not None],
                             self.ww_p, self.bin_width)
        cfg = HistConfig(_capi.MANAGER_MT, 1, float(self.bin_width), int(self.bin_count), 0.0)
        n = r["max_bin"]
        res = {"max_bin": n, "pairs": 0, "aa": r["aa"], "aw": r["aw"], "ww": r["ww"], "tot": r["tot"], "d_axis": r["d_axis"]}
        return CompositeDistanceHistogram(cfg, res, self.ctx)


class BatchedProfiles:
    """Profiles of many independent molecules at once (ausaxs_gpu_batch_*): for every molecule the
    result of ``HistogramManagerMTFFAvg(m).calculate_all()->debye_transform()`` (or FFGrid), from
    one captured graph of shared pair launches.  The reference has no batched form; each molecule's
    result equals its single-structure one."""

    def __init__(self, molecules: Sequence[Molecule], grid: bool = False, bin_width: float = 0.25,
                 bin_count: int = 8000, ctx: Optional[_capi.Context] = None):
        self.molecules = list(molecules)
        self.ctx = ctx or _capi.default_context()
        self.grid = grid
        self.bin_count = bin_count
        manager = _capi.MANAGER_FFGRID if grid else _capi.MANAGER_FFAVG
        self.cfg = HistConfig(manager, 1, float(bin_width), int(bin_count), 0.0)
        parts = [m.compact_ff() for m in self.molecules]
        z = None if grid else [m.get_volume_grid() * RHO_WATER / m.size_atom() if m.size_atom() else 0.0
                               for m in self.molecules]
        self._b = _capi.Batch(self.ctx, self.cfg, [p[0] for p in parts], [p[1] for p in parts],
                              [p[2] for p in parts] if grid else None, z)

    def autotune(self):
        return self._b.autotune()

    def set_molecules(self, molecules: Sequence[Molecule]):
        """Replace every molecule by one with the same atoms and waters in new positions (a new
        conformation or pose; FFAvg batches): the plans and captured graph are kept, the excluded-volume
        charges follow the new volumes."""
        if self.grid:
            raise _capi.AusaxsError(_capi.ERR_ARGUMENT, "new positions need an FFAvg batch")
        molecules = list(molecules)
        if len(molecules) != len(self.molecules):
            raise _capi.AusaxsError(_capi.ERR_ARGUMENT, "set_molecules needs one molecule per structure")
        parts = [m.compact_ff() for m in molecules]
        z = [m.get_volume_grid() * RHO_WATER / m.size_atom() if m.size_atom() else 0.0 for m in molecules]
        self._b.set_points([p[0] for p in parts], [p[1] for p in parts], z)
        self.molecules = molecules

    def debye_transform(self, q=None, cw=1.0, cx=1.0, crho=1.0, dw_atomic=0.0, dw_exv=0.0, grid_width=1.0,
                        precision=1, tolerance=1e-4):
        """[n][nq] I(q) of every molecule: FP64 transform (precision 1), or the exact-accumulation
        tensor-core transform with FP64 for every q whose error bound exceeds tolerance (0 or 2)."""
        q = default_q_axis() if q is None else np.ascontiguousarray(q, np.float64)
        return self._b.profile(q, DebyeParams(cw, cx, crho, dw_atomic, dw_exv, grid_width, precision, tolerance))

    def fp64_columns(self) -> int:
        """(molecule, q) values of the last transform recomputed in FP64."""
        return self._b.fp64_columns()

    def histogram(self, i: int) -> dict:
        """Molecule i's histograms from the last transform: raw aa/aw/ww counts by form factor and axes."""
        r, bufs = self._b.histogram(i, self.bin_count)
        m = r.max_bin
        out = {"max_bin": m, "aa": bufs["aa"][: NFF * NFF * m].reshape(NFF, NFF, m),
               "aw": bufs["aw"][: NFF * m].reshape(NFF, m), "ww": bufs["ww"][:m], "d_axis": bufs["d_axis"][:m]}
        if self.grid:
            out["d_axis_ax"] = bufs["d_axis_ax"][:m]
            out["d_axis_xx"] = bufs["d_axis_xx"][:m]
        return out

    def close(self):
        self._b.close()
