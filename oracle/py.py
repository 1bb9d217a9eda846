"""ctypes front for the oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries sit behind this module:

* ``liboracle.so``   -- the plain-C restatement in ``oracle/oracle.c``;
* ``_ref/libausaxs_ref.so`` -- the reference itself, compiled from its own
  sources by ``oracle/Makefile`` (only present where the reference sources
  were available at build time, or where the built file was carried along).

Only ``tests/``, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg
use this module, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NFF = 15
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def build_oracle() -> str:
    """Compile the C restatement (gcc, no fast-math, no FMA contraction)."""
    out = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "oracle.c")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        L = C.CDLL(path)
        L.oracle_hist_simple.restype = C.c_int64
        L.oracle_hist_simple.argtypes = [_f32p, C.c_int32, _f32p, C.c_int32, C.c_double, C.c_int32, C.c_int,
                                         C.POINTER(C.c_int32), _f64p, _f64p, _f64p, _f64p, _f64p]
        L.oracle_hist_ff.restype = C.c_int64
        L.oracle_hist_ff.argtypes = [C.c_int, _f32p, C.c_int32, _f32p, C.c_int32, _f32p, C.c_int32, C.c_double,
                                     C.c_int32, C.c_double, C.POINTER(C.c_int32), _f64p, _f64p, _f64p, _f64p, _f64p,
                                     _f64p, _f64p]
        L.oracle_debye_ff.restype = None
        L.oracle_debye_ff.argtypes = [C.c_int, _f64p, _f64p, _f64p, C.c_int32, _f64p, _f64p, _f64p, _f64p, C.c_int32,
                                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _f64p,
                                      _f64p]
        L.oracle_debye_simple.restype = None
        L.oracle_debye_simple.argtypes = [_f64p, _f64p, _f64p, C.c_int32, _f64p, _f64p, C.c_int32, C.c_double, _f64p]
        L.oracle_sinqd.restype = None
        L.oracle_sinqd.argtypes = [_f64p, C.c_int32, C.c_int32, _f64p, _f64p, C.c_int32, _f64p]
        L.oracle_ff_raw.restype = C.c_double
        L.oracle_ff_raw.argtypes = [C.c_int, C.c_double]
        L.oracle_ff_exv_volume.restype = C.c_double
        L.oracle_ff_exv_volume.argtypes = [C.c_double, C.c_double]
        L.oracle_linear_lsq.restype = None
        L.oracle_linear_lsq.argtypes = [_f64p, _f64p, _f64p, C.c_int32, _f64p]
        L.oracle_calc_job.restype = C.c_int64
        L.oracle_calc_job.argtypes = [_f32p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                      _f64p, _f64p, _f64p]
        L.oracle_hydrate_axes.restype = None
        L.oracle_hydrate_axes.argtypes = [_f64p, C.c_int64, _f64p]
        L.oracle_hydrate.restype = C.c_int64
        L.oracle_hydrate.argtypes = [_f64p, _i32p, C.c_int64, _f64p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
        _u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        for name in ("oracle_hgrid_add", "oracle_hgrid_remove"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [_u8p, _f64p, _f64p, _i32p, C.c_int64]
        L.oracle_hgrid_hydrate.restype = C.c_int64
        L.oracle_hgrid_hydrate.argtypes = [_u8p, _f64p, _f64p, _i32p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64,
                                           C.c_void_p]
        L.oracle_fit.restype = None
        L.oracle_fit.argtypes = [C.c_int, _f64p, _f64p, _f64p, C.c_int32, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                 C.c_int32, C.c_int, C.c_double, C.c_double, C.c_double, _f64p, C.c_double, _f64p]
        _lib = L
    return _lib


def pack_points(xyz: np.ndarray, fourth: np.ndarray, as_int: bool) -> np.ndarray:
    """float32 [n,4] records {x, y, z, w|ff} as the reference's compact coordinates."""
    n = len(xyz)
    out = np.zeros((n, 4), np.float32)
    out[:, :3] = np.asarray(xyz, np.float64).astype(np.float32)
    if as_int:
        out[:, 3] = np.asarray(fourth, np.int32).view(np.float32)
    else:
        out[:, 3] = np.asarray(fourth, np.float64).astype(np.float32)
    return np.ascontiguousarray(out)


@dataclass
class SimpleHist:
    aa: np.ndarray
    aw: np.ndarray
    ww: np.ndarray
    tot: np.ndarray
    d_axis: np.ndarray
    overflow: int = 0


@dataclass
class FFHist:
    aa: np.ndarray  # [15,15,mb]
    aw: np.ndarray  # [15,mb]
    ww: np.ndarray  # [mb]
    tot: np.ndarray
    d_axis: np.ndarray
    d_axis_ax: Optional[np.ndarray] = None
    d_axis_xx: Optional[np.ndarray] = None
    overflow: int = 0


def hist_simple(atoms4, waters4, bin_width, nbins, weighted=True) -> SimpleHist:
    L = lib()
    mb = C.c_int32(0)
    bufs = [np.zeros(nbins) for _ in range(5)]
    of = L.oracle_hist_simple(np.ascontiguousarray(atoms4, np.float32), len(atoms4),
                              np.ascontiguousarray(waters4, np.float32), len(waters4), bin_width, nbins,
                              int(weighted), C.byref(mb), *bufs)
    m = mb.value
    return SimpleHist(*(b[:m].copy() for b in bufs), overflow=int(of))


def hist_ff(kind, atoms4, waters4, exv4=None, bin_width=0.25, nbins=8000, z_exv=0.0) -> FFHist:
    """kind: 0 FFAvg, 1 FFExplicit, 2 FFGrid."""
    L = lib()
    mb = C.c_int32(0)
    if exv4 is None:
        exv4 = np.zeros((0, 4), np.float32)
    aa = np.zeros(NFF * NFF * nbins)
    aw = np.zeros(NFF * nbins)
    ww, tot, d, dax, dxx = (np.zeros(nbins) for _ in range(5))
    of = L.oracle_hist_ff(kind, np.ascontiguousarray(atoms4, np.float32), len(atoms4),
                          np.ascontiguousarray(waters4, np.float32), len(waters4),
                          np.ascontiguousarray(exv4, np.float32), len(exv4), bin_width, nbins, z_exv, C.byref(mb),
                          aa, aw, ww, tot, d, dax, dxx)
    m = mb.value
    return FFHist(aa[: NFF * NFF * m].reshape(NFF, NFF, m).copy(), aw[: NFF * m].reshape(NFF, m).copy(), ww[:m].copy(),
                  tot[:m].copy(), d[:m].copy(), dax[:m].copy() if kind == 2 else None,
                  dxx[:m].copy() if kind == 2 else None, overflow=int(of))


def debye_ff(kind, h: FFHist, q, cw=1.0, cx=1.0, crho=1.0, dw_atomic=0.0, dw_exv=0.0, grid_width=1.0):
    L = lib()
    q = np.ascontiguousarray(q, np.float64)
    nq = len(q)
    mb = len(h.d_axis)
    prof = np.zeros(6 * nq)
    I = np.zeros(nq)
    dax = h.d_axis_ax if h.d_axis_ax is not None else h.d_axis
    dxx = h.d_axis_xx if h.d_axis_xx is not None else h.d_axis
    L.oracle_debye_ff(kind, np.ascontiguousarray(h.aa.reshape(-1)), np.ascontiguousarray(h.aw.reshape(-1)),
                      np.ascontiguousarray(h.ww), mb, np.ascontiguousarray(h.d_axis), np.ascontiguousarray(dax),
                      np.ascontiguousarray(dxx), q, nq, cw, cx, crho, dw_atomic, dw_exv, grid_width, prof, I)
    return I, prof.reshape(6, nq)


# The reference's search limits per parameter (ICompositeDistanceHistogram.h:70,
# ICompositeDistanceHistogramExv.cpp:8-12): cw, cx, crho, atomic and exv Debye-Waller.
FIT_LIMITS = {0: (0.0, 10.0), 1: (0.92, 1.08), 2: (0.5, 2.0), 3: (0.0, 5.0), 4: (0.0, 5.0)}


def fit(kind, h, q, y, sigma, param=0, lo=None, hi=None, tol=1e-4, base=(1.0, 1.0, 1.0, 0.0, 0.0), grid_width=1.0):
    """SmartFitter::fit with the Golden minimiser over one parameter (kind 3: Simple histogram).
    Returns (value, a, b, chi2, evaluations)."""
    L = lib()
    f = L.oracle_fit
    lo = FIT_LIMITS[param][0] if lo is None else lo
    hi = FIT_LIMITS[param][1] if hi is None else hi
    q, y, sigma = (np.ascontiguousarray(x, np.float64) for x in (q, y, sigma))
    out = np.zeros(5)
    base = np.ascontiguousarray(base, np.float64)
    if kind == 3:
        aa, aw, ww = (np.ascontiguousarray(x) for x in (h.aa, h.aw, h.ww))
        dax = dxx = np.ascontiguousarray(h.d_axis)
    else:
        aa, aw, ww = np.ascontiguousarray(h.aa.reshape(-1)), np.ascontiguousarray(h.aw.reshape(-1)), np.ascontiguousarray(h.ww)
        dax = np.ascontiguousarray(h.d_axis_ax if h.d_axis_ax is not None else h.d_axis)
        dxx = np.ascontiguousarray(h.d_axis_xx if h.d_axis_xx is not None else h.d_axis)
    f(int(kind), aa, aw, ww, len(h.d_axis), np.ascontiguousarray(h.d_axis), dax, dxx, q, y, sigma, len(q), int(param),
      float(lo), float(hi), float(tol), base, float(grid_width), out)
    return out[0], out[1], out[2], out[3], int(out[4])


def debye_simple(h: SimpleHist, q, cw=1.0):
    L = lib()
    q = np.ascontiguousarray(q, np.float64)
    I = np.zeros(len(q))
    L.oracle_debye_simple(h.aa, h.aw, h.ww, len(h.d_axis), np.ascontiguousarray(h.d_axis), q, len(q), cw, I)
    return I


def sinqd(p, d_axis, q):
    L = lib()
    p = np.ascontiguousarray(np.atleast_2d(p), np.float64)
    out = np.zeros((p.shape[0], len(q)))
    L.oracle_sinqd(p, p.shape[0], p.shape[1], np.ascontiguousarray(d_axis, np.float64),
                   np.ascontiguousarray(q, np.float64), len(q), out)
    return out


def ff_raw(t, q):
    return np.array([lib().oracle_ff_raw(int(t), float(x)) for x in np.atleast_1d(q)])


def grid_exv(xyz, ff, waters=None):
    """Grid excluded-volume dummies of the expanded molecular grid (RawGridExv::create): [n, 3], volume."""
    L = lib()
    f = L.oracle_grid_exv
    f.restype = C.c_int64
    f.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_double)]
    a = np.ascontiguousarray(np.column_stack([np.asarray(xyz, float).reshape(-1, 3), np.asarray(ff, float)]))
    w = np.ascontiguousarray(np.zeros((0, 3)) if waters is None else np.asarray(waters, float).reshape(-1, 3))
    vol = C.c_double(0)
    n = f(a.ctypes.data, len(a), w.ctypes.data, len(w), None, 0, C.byref(vol))
    out = np.zeros((max(1, n), 3))
    f(a.ctypes.data, len(a), w.ctypes.data, len(w), out.ctypes.data, n, C.byref(vol))
    return out[:n], vol.value


def linear_lsq(data, model, err):
    out = np.zeros(5)
    lib().oracle_linear_lsq(np.ascontiguousarray(data, np.float64), np.ascontiguousarray(model, np.float64),
                            np.ascontiguousarray(err, np.float64), len(data), out)
    return out


# ---------------------------------------------------------------------------
# The reference compiled from source (oracle/_ref/libausaxs_ref.so)
# ---------------------------------------------------------------------------

def ref_path() -> str:
    """The compiled reference; AUSAXS_REF_LIB=libausaxs_ref_gpu.so selects its adapter build (the
    reference's Simple, partial and symmetry managers over the device calculator, and the device FFAvg
    manager: oracle/Makefile target `adapter`)."""
    return os.path.join(HERE, "_ref", os.environ.get("AUSAXS_REF_LIB", "libausaxs_ref.so"))


def ref_read_structure(path: str, implicit_h: int = -1, center: int = -1):
    """A structure file read by the reference's own reader: (xyz [n,3], weights [n], ff [n] int,
    waters [m,3], water weights [m])."""
    L = ref()
    f = L.ref_read_structure
    f.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_int,
                  C.POINTER(C.c_int)]
    na, nw = C.c_int(), C.c_int()
    if f(path.encode(), implicit_h, center, None, 0, C.byref(na), None, 0, C.byref(nw)):
        raise RuntimeError(L.ref_last_error().decode())
    a = np.zeros((max(1, na.value), 5))
    w = np.zeros((max(1, nw.value), 4))
    if f(path.encode(), implicit_h, center, a.ctypes.data, na.value, C.byref(na), w.ctypes.data, nw.value, C.byref(nw)):
        raise RuntimeError(L.ref_last_error().decode())
    a, w = a[: na.value], w[: nw.value]
    return a[:, :3].copy(), a[:, 3].copy(), a[:, 4].astype(np.int32), w[:, :3].copy(), w[:, 3].copy()


def ref_grid_exv(xyz, ff, waters=None):
    """RawGridExv::create of the reference on the expanded grid: dummies [n, 3], volume."""
    L = ref()
    f = L.ref_grid_exv
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                  C.POINTER(C.c_double)]
    a = np.ascontiguousarray(np.column_stack([np.asarray(xyz, float).reshape(-1, 3), np.asarray(ff, float)]))
    w = np.ascontiguousarray(np.zeros((0, 3)) if waters is None else np.asarray(waters, float).reshape(-1, 3))
    n, vol = C.c_int(), C.c_double()
    if f(a.ctypes.data, len(a), w.ctypes.data, len(w), None, 0, C.byref(n), C.byref(vol)):
        raise RuntimeError(L.ref_last_error().decode())
    out = np.zeros((max(1, n.value), 3))
    if f(a.ctypes.data, len(a), w.ctypes.data, len(w), out.ctypes.data, n.value, C.byref(n), C.byref(vol)):
        raise RuntimeError(L.ref_last_error().decode())
    return out[: n.value], vol.value


def ref_grid_exv_seconds(xyz, ff, waters=None) -> tuple:
    """Wall time of one reference RawGridExv::create on a fresh molecule (grid creation, expansion and
    sweep; the dummies are counted, not copied out): (seconds, dummy count, volume)."""
    import time

    L = ref()
    f = L.ref_grid_exv
    f.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                  C.POINTER(C.c_double)]
    a = np.ascontiguousarray(np.column_stack([np.asarray(xyz, float).reshape(-1, 3), np.asarray(ff, float)]))
    w = np.ascontiguousarray(np.zeros((0, 3)) if waters is None else np.asarray(waters, float).reshape(-1, 3))
    n, vol = C.c_int(), C.c_double()
    t0 = time.perf_counter()
    rc = f(a.ctypes.data, len(a), w.ctypes.data, len(w), None, 0, C.byref(n), C.byref(vol))
    t = time.perf_counter() - t0
    if rc:
        raise RuntimeError(L.ref_last_error().decode())
    return t, n.value, vol.value


def ref_available() -> bool:
    return os.path.exists(ref_path())


def ref(threads: int = 0):
    """Load the compiled reference once; threads sizes its global pool (first call only)."""
    global _ref
    if _ref is None:
        R = C.CDLL(ref_path())
        vp = C.c_void_p
        R.ref_last_error.restype = C.c_char_p
        R.ref_init.argtypes = [C.c_int]
        R.ref_set_axes.argtypes = [C.c_double, C.c_int, C.c_double, C.c_double]
        R.ref_set_simple_exv.argtypes = [C.c_int]
        R.ref_molecule_new.restype = vp
        R.ref_molecule_new.argtypes = [_f64p, C.c_int, _f64p, C.c_int, _i32p, C.c_int, C.c_double]
        R.ref_molecule_free.argtypes = [vp]
        R.ref_body_move.argtypes = [vp, C.c_int, _f64p, _f64p]
        R.ref_body_add_symmetry.argtypes = [vp, C.c_int, C.c_char_p, C.c_double, C.c_double]
        R.ref_adapter_build.restype = C.c_int
        R.ref_body_coords.argtypes = [vp, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        R.ref_body_move_in_grid.argtypes = [vp, C.c_int, _f64p, _f64p]
        R.ref_hydrate.argtypes = [vp, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p,
                                  C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p]
        R.ref_manager_set.argtypes = [vp, C.c_int, C.c_int, _f64p, C.c_int]
        R.ref_manager_calculate.restype = vp
        R.ref_manager_calculate.argtypes = [vp, C.POINTER(C.c_double)]
        R.ref_hist_free.argtypes = [vp]
        R.ref_hist_bins.argtypes = [vp]
        R.ref_hist_total.argtypes = [vp, _f64p, _f64p]
        R.ref_hist_simple.argtypes = [vp, _f64p, _f64p, _f64p]
        R.ref_hist_ff.argtypes = [vp, _f64p, _f64p, _f64p]
        R.ref_hist_grid_axes.argtypes = [vp, _f64p, _f64p]
        R.ref_hist_grid_axis_sizes.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        R.ref_debye.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _f64p, _f64p, _f64p,
                                C.POINTER(C.c_int), C.POINTER(C.c_double)]
        R.ref_exact_debye.argtypes = [vp, _f64p, C.c_int, _f64p]
        R.ref_linear_lsq.argtypes = [_f64p, _f64p, _f64p, C.c_int, _f64p]
        R.ref_fit.argtypes = [vp, C.c_int, _f64p, _f64p, _f64p, C.c_int, _f64p]
        R.ref_calculator.argtypes = [_f64p, _i32p, C.c_int, C.c_int, _i32p, _i32p, _i32p, _i32p,
                                     C.POINTER(C.c_int), _i32p, _f64p]
        n = threads if threads > 0 else max(1, (os.cpu_count() or 2) - 1)
        _check(R, R.ref_init(n))
        _ref = R
    return _ref


def _check(R, rc):
    if rc != 0:
        raise RuntimeError("reference: " + R.ref_last_error().decode())


MANAGERS = {"single": 0, "mt": 1, "ffavg": 2, "ffexplicit": 3, "ffgrid": 4, "partial": 5, "symmetry": 6,
            "gpu_ffavg": 7}


class RefMolecule:
    """A reference data::Molecule built from arrays (atoms: x y z w ff; waters: x y z w)."""

    def __init__(self, atoms_xyz, atoms_w, atoms_ff, waters_xyz, waters_w, body_sizes=None, volume=-1.0):
        R = ref()
        na = len(atoms_xyz)
        a = np.zeros((na, 5))
        a[:, :3] = atoms_xyz
        a[:, 3] = atoms_w
        a[:, 4] = atoms_ff
        nw = len(waters_xyz)
        w = np.zeros((max(nw, 1), 4))
        if nw:
            w[:nw, :3] = waters_xyz
            w[:nw, 3] = waters_w
        bs = np.asarray(body_sizes if body_sizes is not None else [na], np.int32)
        self.h = R.ref_molecule_new(np.ascontiguousarray(a.reshape(-1)) if na else np.zeros(5), na,
                                    np.ascontiguousarray(w.reshape(-1)), nw, bs, len(bs), float(volume))
        if not self.h:
            raise RuntimeError("reference: " + R.ref_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_molecule_free(self.h)
            self.h = None

    def set_manager(self, name, weighted_bins=True, exv_xyz=None):
        R = ref()
        x = np.zeros(3) if exv_xyz is None or len(exv_xyz) == 0 else np.ascontiguousarray(np.asarray(exv_xyz, np.float64).reshape(-1))
        nx = 0 if exv_xyz is None else len(exv_xyz)
        _check(R, R.ref_manager_set(self.h, MANAGERS[name], int(weighted_bins), x, nx))

    def body_coords(self, body):
        """The body's current atom coordinates (after any moves), [n, 3] float64; body = -1: the
        molecule's waters, which their owning body carries along when it moves."""
        R = ref()
        n = C.c_int(0)
        _check(R, R.ref_body_coords(self.h, body, None, C.byref(n)))
        out = np.zeros((max(1, n.value), 3))
        _check(R, R.ref_body_coords(self.h, body, out.ctypes.data, C.byref(n)))
        return out[:n.value]

    def hydrate(self, noise=None, fresh_grid=True, n_bodies=1):
        """Molecule::generate_new_hydration() (RadialHydration, no culling) with the noise generator
        reading the rows of `noise` ([n, 3], zero when None).  Returns (grid member atoms in visiting
        order [n, 4] {x, y, z, ff}, waters [m, 3] in body order, waters per body, grid axes [9]
        {min xyz, max xyz, bins xyz}, seconds)."""
        import time

        R = ref()
        nz = None if noise is None else np.ascontiguousarray(np.asarray(noise, np.float64).reshape(-1, 3))
        na, nw = C.c_int(0), C.c_int(0)
        per_body = np.zeros(max(1, n_bodies), np.int32)
        axes = np.zeros(9)
        t0 = time.perf_counter()
        _check(R, R.ref_hydrate(self.h, None if nz is None else nz.ctypes.data, 0 if nz is None else len(nz),
                                int(fresh_grid), None, 0, C.byref(na), None, 0, C.byref(nw), per_body.ctypes.data,
                                axes.ctypes.data))
        secs = time.perf_counter() - t0
        atoms = np.zeros((max(1, na.value), 4))
        waters = np.zeros((max(1, nw.value), 3))
        # the second call regenerates with the same noise rows; the result is the same hydration
        _check(R, R.ref_hydrate(self.h, None if nz is None else nz.ctypes.data, 0 if nz is None else len(nz), 0,
                                atoms.ctypes.data, len(atoms), C.byref(na), waters.ctypes.data, len(waters),
                                C.byref(nw), per_body.ctypes.data, axes.ctypes.data))
        return atoms[:na.value], waters[:nw.value], per_body[:n_bodies].copy(), axes, secs

    def move_body_in_grid(self, body, Rm, t):
        """The rigid-body transforms' move: the body leaves the grid, moves and is appended back."""
        R = ref()
        _check(R, R.ref_body_move_in_grid(self.h, body, np.ascontiguousarray(np.asarray(Rm, np.float64).reshape(9)),
                                          np.ascontiguousarray(np.asarray(t, np.float64).reshape(3))))

    def add_symmetry(self, body, name, translation, rotation=0.0):
        """A predefined symmetry of the reference (symmetry::create(name)) on a body."""
        _check(ref(), ref().ref_body_add_symmetry(self.h, body, name.encode(), float(translation), float(rotation)))

    def move_body(self, body, Rm, t):
        R = ref()
        _check(R, R.ref_body_move(self.h, body, np.ascontiguousarray(np.asarray(Rm, np.float64).reshape(9)),
                                  np.ascontiguousarray(np.asarray(t, np.float64).reshape(3))))

    def calculate(self):
        R = ref()
        secs = C.c_double(0)
        hp = R.ref_manager_calculate(self.h, C.byref(secs))
        if not hp:
            raise RuntimeError("reference: " + R.ref_last_error().decode())
        return RefHist(hp, secs.value)

    def exact_debye(self, q):
        R = ref()
        q = np.ascontiguousarray(q, np.float64)
        out = np.zeros(len(q))
        _check(R, R.ref_exact_debye(self.h, q, len(q), out))
        return out


class RefHist:
    def __init__(self, h, seconds):
        self.h = h
        self.seconds = seconds

    def __del__(self):
        if getattr(self, "h", None) and _ref is not None:
            _ref.ref_hist_free(self.h)
            self.h = None

    @property
    def bins(self):
        return ref().ref_hist_bins(self.h)

    def total(self):
        n = self.bins
        c, d = np.zeros(n), np.zeros(n)
        _check(ref(), ref().ref_hist_total(self.h, c, d))
        return c, d

    def simple(self):
        n = self.bins
        a, b, c = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(ref(), ref().ref_hist_simple(self.h, a, b, c))
        return a, b, c

    def ff(self):
        n = self.bins
        a, b, c = np.zeros(NFF * NFF * n), np.zeros(NFF * n), np.zeros(n)
        _check(ref(), ref().ref_hist_ff(self.h, a, b, c))
        return a.reshape(NFF, NFF, n), b.reshape(NFF, n), c

    def grid_axes(self):
        na, nx = C.c_int(0), C.c_int(0)
        _check(ref(), ref().ref_hist_grid_axis_sizes(self.h, C.byref(na), C.byref(nx)))
        a, x = np.zeros(na.value), np.zeros(nx.value)
        _check(ref(), ref().ref_hist_grid_axes(self.h, a, x))
        return a, x

    def fit(self, param: int, q, I, sigma):
        """fitter::SmartFitter(data, histogram).fit() with one enabled parameter (consumes the
        histogram): (value, a, b, chi2, evaluations)."""
        R = ref()
        out = np.zeros(6)
        q, I, sigma = (np.ascontiguousarray(x, np.float64) for x in (q, I, sigma))
        _check(R, R.ref_fit(self.h, int(param), q, I, sigma, len(q), out))
        self.fit_seconds = out[5]
        return out[0], out[1], out[2], out[3], int(out[4])

    def debye(self, cw=1.0, cx=1.0, crho=1.0, dw_atomic=0.0, dw_exv=0.0):
        R = ref()
        q, I, prof = np.zeros(200), np.zeros(200), np.zeros(6 * 200)
        nq = C.c_int(0)
        secs = C.c_double(0)
        _check(R, R.ref_debye(self.h, cw, cx, crho, dw_atomic, dw_exv, q, I, prof, C.byref(nq), C.byref(secs)))
        n = nq.value
        return q[:n].copy(), I[:n].copy(), prof[: 6 * n].reshape(6, n).copy(), secs.value


def calculator(sets, jobs, bin_width, nbins):
    """SimpleCalculator<true, false> restated: sets = list of [n, 4] float32 {x, y, z, w} records;
    jobs = [(a, b or None, scaling, merge_id)].  Returns {(is_cross, merge_id): (value, count, dsum)}."""
    L = lib()
    out = {}
    n_results = [0, 0]  # results of each kind so far
    for a, b, scaling, merge in jobs:
        kind = 0 if b is None else 1
        if merge == -1:  # a result of its own, with id = the number of results of this kind (SimpleCalculator.h:100-109)
            merge = n_results[kind]
        key = (kind, merge)
        if key not in out:
            n_results[kind] += 1
            out[key] = tuple(np.zeros(nbins) for _ in range(3))
        v, c, d = out[key]
        A = np.ascontiguousarray(sets[a], np.float32)
        B = None if b is None else np.ascontiguousarray(sets[b], np.float32)
        L.oracle_calc_job(A, len(A), None if B is None else B.ctypes.data, 0 if B is None else len(B), int(scaling),
                          float(bin_width), int(nbins), v, c, d)
    return out


HYDRATE_DIRECTIONS = 26


def hydrate_noise(n_candidates: int, seed: int) -> np.ndarray:
    """A reproducible noise table for the hydration tests, [n, 3] in (-0.75, 0.75): a multiplicative
    integer hash of (seed, row, component) scaled to the range, exact in double on every platform."""
    k = np.arange(3 * n_candidates, dtype=np.uint64) + np.uint64(seed) * np.uint64(0x9E3779B1)
    h = (k * np.uint64(2654435761) + np.uint64(seed)) % np.uint64(1 << 32)
    h = (h ^ (h >> np.uint64(15))) * np.uint64(2246822519) % np.uint64(1 << 32)
    return ((h.astype(np.float64) / 4294967296.0) - 0.5).reshape(-1, 3) * 1.5


def hydrate_axes(xyz):
    """Grid axes {min x, y, z, bins x, y, z} of Grid(bodies) over the atoms alone."""
    a = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    out = np.zeros(6)
    lib().oracle_hydrate_axes(a, len(a), out)
    return out


def hydrate(xyz, ff, axes=None, noise=None):
    """RadialHydration restated (oracle_hydrate): waters [m, 3] and their candidate indices
    (atom * 26 + direction), atoms in the order the generator visits them."""
    a = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(ff, np.int32).reshape(-1))
    ax = hydrate_axes(a) if axes is None else np.ascontiguousarray(np.asarray(axes, np.float64)[:6])
    nz = None if noise is None else np.ascontiguousarray(np.asarray(noise, np.float64).reshape(-1, 3))
    if nz is not None and len(nz) < HYDRATE_DIRECTIONS * len(a):
        nz = np.vstack([nz, np.zeros((HYDRATE_DIRECTIONS * len(a) - len(nz), 3))])
    cap = HYDRATE_DIRECTIONS * len(a) + 1
    out = np.zeros((cap, 3))
    cand = np.zeros(cap, np.int64)
    m = lib().oracle_hydrate(a, f, len(a), ax, None if nz is None else nz.ctypes.data, out.ctypes.data, cap,
                             cand.ctypes.data)
    if m < 0:
        raise RuntimeError(f"oracle_hydrate failed ({m})")
    return out[:m], cand[:m]


class HydrationGrid:
    """The oracle's hydration grid kept across calls, as the reference keeps a molecule's grid::Grid:
    add(xyz, ff) = Grid::add with the volume expansion, remove(xyz, ff) = Grid::remove of atoms at
    those (current) coordinates, hydrate(xyz, ff, noise) = the generation over the grid's members in
    the order given (oracle_hgrid_*)."""

    def __init__(self, axes):
        self.axes = np.ascontiguousarray(np.asarray(axes, np.float64)[:6])
        self.state = np.zeros(int(np.prod(self.axes[3:].astype(np.int64))), np.uint8)

    @staticmethod
    def _in(xyz, ff):
        return (np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3)),
                np.ascontiguousarray(np.asarray(ff, np.int32).reshape(-1)))

    def add(self, xyz, ff):
        a, f = self._in(xyz, ff)
        lib().oracle_hgrid_add(self.state, self.axes, a, f, len(a))

    def remove(self, xyz, ff):
        a, f = self._in(xyz, ff)
        lib().oracle_hgrid_remove(self.state, self.axes, a, f, len(a))

    def hydrate(self, xyz, ff, noise=None):
        a, f = self._in(xyz, ff)
        nz = None if noise is None else np.ascontiguousarray(np.asarray(noise, np.float64).reshape(-1, 3))
        cap = HYDRATE_DIRECTIONS * len(a) + 1
        out = np.zeros((cap, 3))
        cand = np.zeros(cap, np.int64)
        m = lib().oracle_hgrid_hydrate(self.state, self.axes, a, f, len(a), None if nz is None else nz.ctypes.data,
                                       out.ctypes.data, cap, cand.ctypes.data)
        if m < 0:
            raise RuntimeError(f"oracle_hgrid_hydrate failed ({m})")
        return out[:m], cand[:m]


def ref_calculator(sets, jobs):
    """The reference's SimpleCalculator<true, false> on the same jobs (bins: settings::axes)."""
    R = ref()
    pts = np.ascontiguousarray(np.concatenate([np.asarray(s, np.float64).reshape(-1, 4) for s in sets]))
    off = np.zeros(len(sets) + 1, np.int32)
    off[1:] = np.cumsum([len(s) for s in sets])
    ja = np.array([j[0] for j in jobs], np.int32)
    jb = np.array([-1 if j[1] is None else j[1] for j in jobs], np.int32)
    sc = np.array([j[2] for j in jobs], np.int32)
    mg = np.array([j[3] for j in jobs], np.int32)
    nbins = R.ref_hist_bins_setting() if hasattr(R, "ref_hist_bins_setting") else 8000
    n = C.c_int(0)
    keys = np.zeros(2 * len(jobs), np.int32)
    out = np.zeros(3 * len(jobs) * nbins)
    _check(R, R.ref_calculator(pts, off, len(sets), len(jobs), ja, jb, sc, mg, C.byref(n), keys, out))
    res = {}
    for r in range(n.value):
        v = out[3 * r * nbins:(3 * r + 3) * nbins].reshape(3, nbins)
        res[(int(keys[2 * r]), int(keys[2 * r + 1]))] = (v[0].copy(), v[1].copy(), v[2].copy())
    return res


def ref_set_axes(bin_width=0.25, bin_count=8000, qmin=1e-4, qmax=0.5):
    R = ref()
    _check(R, R.ref_set_axes(bin_width, bin_count, qmin, qmax))


def ref_set_simple_exv(enable: bool):
    R = ref()
    _check(R, R.ref_set_simple_exv(int(enable)))


def ref_linear_lsq(data, model, err):
    R = ref()
    out = np.zeros(5)
    _check(R, R.ref_linear_lsq(np.ascontiguousarray(data, np.float64), np.ascontiguousarray(model, np.float64),
                               np.ascontiguousarray(err, np.float64), len(data), out))
    return out
