"""ctypes binding of the C ABI in include/ausaxs_b200.h.

The library is the in-tree ``ausaxs_b200/_lib/libausaxs_b200.so`` built by ``ausaxs_b200.build``.
There is no CPU fallback: importing a GPU entry point without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libausaxs_b200.so")

OK = 0
ERR_ARGUMENT = 1
ERR_CUDA = 2
ERR_BIN_OVERFLOW = 3
ERR_FORM_FACTOR = 4
ERR_CAPACITY = 5
ERR_TIMEOUT = 6
ERR_NOT_FOUND = 7

MANAGER_MT = 1
MANAGER_FFAVG = 2
MANAGER_FFEXPLICIT = 3
MANAGER_FFGRID = 4

# every symbol include/ausaxs_b200.h and include/ausaxs_b200_diag.h declare
EXPORTED = [
    "ausaxs_gpu_ctx_create", "ausaxs_gpu_ctx_destroy", "ausaxs_gpu_ctx_set_stream", "ausaxs_gpu_ctx_launch_count",
    "ausaxs_gpu_last_error", "ausaxs_gpu_ctx_enable_timing", "ausaxs_gpu_ctx_kernel_time",
    "ausaxs_gpu_ctx_fp64_columns", "ausaxs_gpu_ctx_tc_error_estimate", "ausaxs_gpu_histogram", "ausaxs_gpu_debye", "ausaxs_gpu_profile",
    "ausaxs_gpu_structure_create", "ausaxs_gpu_structure_destroy", "ausaxs_gpu_structure_profile",
    "ausaxs_gpu_structure_histogram", "ausaxs_gpu_histogram_mt_noalloc", "ausaxs_gpu_linear_lsq", "ausaxs_gpu_grid_exv",
    "ausaxs_gpu_fit", "ausaxs_gpu_structure_fit", "ausaxs_gpu_hydrate", "ausaxs_gpu_hydrate_device", "ausaxs_hydrate_axes",
    "ausaxs_gpu_ctx_hydration_stats",
    "ausaxs_gpu_hydration_grid_create", "ausaxs_gpu_hydration_grid_destroy", "ausaxs_gpu_hydration_grid_add",
    "ausaxs_gpu_hydration_grid_remove", "ausaxs_gpu_hydration_grid_hydrate",
    "ausaxs_gpu_calculator_create", "ausaxs_gpu_calculator_destroy", "ausaxs_gpu_calculator_enqueue_self",
    "ausaxs_gpu_calculator_enqueue_cross", "ausaxs_gpu_calculator_run", "ausaxs_gpu_calculator_result_ids",
    "ausaxs_gpu_calculator_result",
    "ausaxs_gpu_batch_create", "ausaxs_gpu_batch_destroy", "ausaxs_gpu_batch_autotune", "ausaxs_gpu_batch_candidate",
    "ausaxs_gpu_batch_profile_device", "ausaxs_gpu_batch_profile", "ausaxs_gpu_batch_pair_time",
    "ausaxs_gpu_batch_histogram", "ausaxs_gpu_batch_set_points", "ausaxs_gpu_batch_fp64_columns", "ausaxs_gpu_smem_atomic_rate",
    "ausaxs_gpu_server_create", "ausaxs_gpu_server_set_policy", "ausaxs_gpu_server_destroy", "ausaxs_gpu_server_admit", "ausaxs_gpu_server_release",
    "ausaxs_gpu_server_usage", "ausaxs_gpu_server_submit", "ausaxs_gpu_server_poll", "ausaxs_gpu_server_wait",
    "ausaxs_gpu_server_completed", "ausaxs_gpu_server_launch_count", "ausaxs_gpu_server_body_center", "ausaxs_gpu_server_coordinates", "ausaxs_gpu_server_histogram",
]


class AusaxsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class HistConfig(C.Structure):
    _fields_ = [("manager", C.c_int32), ("weighted_bins", C.c_int32), ("bin_width", C.c_double),
                ("bin_count", C.c_int32), ("z_exv", C.c_double)]


class HistResult(C.Structure):
    _fields_ = [("max_bin", C.c_int32), ("pairs", C.c_int64), ("overflow_pairs", C.c_int64),
                ("aa", C.POINTER(C.c_double)), ("aw", C.POINTER(C.c_double)), ("ww", C.POINTER(C.c_double)),
                ("tot", C.POINTER(C.c_double)), ("d_axis", C.POINTER(C.c_double)),
                ("d_axis_ax", C.POINTER(C.c_double)), ("d_axis_xx", C.POINTER(C.c_double))]


class DebyeParams(C.Structure):
    _fields_ = [("cw", C.c_double), ("cx", C.c_double), ("crho", C.c_double), ("dw_atomic", C.c_double),
                ("dw_exv", C.c_double), ("grid_width", C.c_double), ("precision", C.c_int32),
                ("tolerance", C.c_double)]


class FitOptions(C.Structure):
    _fields_ = [("parameter", C.c_int32), ("lo", C.c_double), ("hi", C.c_double), ("tolerance", C.c_double)]


class FitResult(C.Structure):
    _fields_ = [("value", C.c_double), ("a", C.c_double), ("b", C.c_double), ("a_err", C.c_double),
                ("b_err", C.c_double), ("chi2", C.c_double), ("evaluations", C.c_int32)]


# fitted-parameter indices of ausaxs_fit_options (SmartFitter's EnabledFitParameters order)
FIT_PARAMETERS = {"cw": 0, "cx": 1, "crho": 2, "dw_atomic": 3, "dw_exv": 4}

_lib = None
_lock = threading.Lock()


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m ausaxs_b200.build` (needs nvcc)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        f32 = C.POINTER(C.c_float)
        f64 = C.POINTER(C.c_double)
        L.ausaxs_gpu_last_error.restype = C.c_char_p
        L.ausaxs_gpu_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.ausaxs_gpu_ctx_destroy.argtypes = [vp]
        L.ausaxs_gpu_ctx_set_stream.argtypes = [vp, vp]
        L.ausaxs_gpu_ctx_launch_count.argtypes = [vp]
        L.ausaxs_gpu_ctx_launch_count.restype = C.c_int64
        L.ausaxs_gpu_ctx_enable_timing.argtypes = [vp, C.c_int32]
        L.ausaxs_gpu_ctx_kernel_time.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.ausaxs_gpu_ctx_fp64_columns.argtypes = [vp, C.POINTER(C.c_int32)]
        L.ausaxs_gpu_ctx_tc_error_estimate.argtypes = [vp, C.POINTER(C.c_double), C.c_int32]
        L.ausaxs_gpu_histogram.argtypes = [vp, C.POINTER(HistConfig), f32, C.c_int32, f32, C.c_int32, f32, C.c_int32,
                                           C.POINTER(HistResult)]
        L.ausaxs_gpu_debye.argtypes = [vp, C.POINTER(HistConfig), C.POINTER(HistResult), f64, C.c_int32,
                                       C.POINTER(DebyeParams), f64, f64]
        L.ausaxs_gpu_profile.argtypes = [vp, C.POINTER(HistConfig), f32, C.c_int32, f32, C.c_int32, f32, C.c_int32,
                                         f64, C.c_int32, C.POINTER(DebyeParams), f64, f64]
        L.ausaxs_gpu_structure_create.argtypes = [vp, C.c_int32, f32, C.c_int32, f32, C.c_int32, f32, C.c_int32,
                                                  C.c_int32, C.POINTER(vp)]
        L.ausaxs_gpu_structure_destroy.argtypes = [vp]
        L.ausaxs_gpu_structure_profile.argtypes = [vp, vp, C.POINTER(HistConfig), f64, C.c_int32,
                                                   C.POINTER(DebyeParams), f64, f64]
        L.ausaxs_gpu_structure_histogram.argtypes = [vp, vp, C.POINTER(HistConfig), C.POINTER(HistResult)]
        L.ausaxs_gpu_linear_lsq.argtypes = [vp, f64, f64, f64, C.c_int32, f64]
        L.ausaxs_gpu_fit.argtypes = [vp, C.POINTER(HistConfig), C.POINTER(HistResult), f64, f64, f64, C.c_int32,
                                     C.POINTER(DebyeParams), C.POINTER(FitOptions), C.POINTER(FitResult), f64]
        L.ausaxs_gpu_structure_fit.argtypes = [vp, vp, C.POINTER(HistConfig), f64, f64, f64, C.c_int32,
                                               C.POINTER(DebyeParams), C.POINTER(FitOptions), C.POINTER(FitResult), f64]
        i32p = C.POINTER(C.c_int32)
        L.ausaxs_gpu_calculator_create.argtypes = [vp, C.c_double, C.c_int32, C.POINTER(vp)]
        L.ausaxs_gpu_calculator_destroy.argtypes = [vp]
        L.ausaxs_gpu_calculator_enqueue_self.argtypes = [vp, f32, C.c_int32, C.c_int32, C.c_int32, i32p]
        L.ausaxs_gpu_calculator_enqueue_cross.argtypes = [vp, f32, C.c_int32, f32, C.c_int32, C.c_int32, C.c_int32, i32p]
        L.ausaxs_gpu_calculator_run.argtypes = [vp, i32p, i32p]
        L.ausaxs_gpu_calculator_result_ids.argtypes = [vp, C.c_int32, i32p, C.c_int32, i32p]
        L.ausaxs_gpu_calculator_result.argtypes = [vp, C.c_int32, C.c_int32, f64, f64, f64]
        L.ausaxs_gpu_grid_exv.argtypes = [vp, f32, C.c_int32, f32, C.c_int32, C.c_int32, f32, C.c_int64,
                                          C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        i64 = C.POINTER(C.c_int64)
        i32 = C.POINTER(C.c_int32)
        L.ausaxs_gpu_batch_create.argtypes = [vp, C.POINTER(HistConfig), C.c_int32, f32, i64, f32, i64, f32, i64, f64,
                                              C.c_int32, C.POINTER(vp)]
        L.ausaxs_gpu_batch_destroy.argtypes = [vp]
        L.ausaxs_gpu_batch_autotune.argtypes = [vp, i32, f64, C.c_int32]
        L.ausaxs_gpu_batch_candidate.argtypes = [C.c_int32, i32, i32, i32, i32]
        L.ausaxs_gpu_batch_profile_device.argtypes = [vp, f64, C.c_int32, C.POINTER(DebyeParams), f64]
        L.ausaxs_gpu_batch_profile.argtypes = [vp, f64, C.c_int32, C.POINTER(DebyeParams), f64]
        L.ausaxs_gpu_batch_pair_time.argtypes = [vp, f64]
        L.ausaxs_gpu_batch_histogram.argtypes = [vp, C.c_int32, C.POINTER(HistResult)]
        L.ausaxs_gpu_batch_set_points.argtypes = [vp, f32, f32, f64, C.c_int32]
        L.ausaxs_gpu_batch_fp64_columns.argtypes = [vp, i64]
        L.ausaxs_gpu_smem_atomic_rate.argtypes = [C.c_int32, C.c_int32, f64, f64]
        L.ausaxs_gpu_server_create.argtypes = [C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.POINTER(vp)]
        L.ausaxs_gpu_server_destroy.argtypes = [vp]
        L.ausaxs_gpu_server_set_policy.argtypes = [vp, C.c_int32]
        L.ausaxs_gpu_server_admit.argtypes = [vp, C.POINTER(HistConfig), C.c_int32, f32, i64, f32, i64, C.c_double,
                                              f64, C.c_int32, C.POINTER(DebyeParams), f64, f64, i32, i64]
        L.ausaxs_gpu_server_release.argtypes = [vp, C.c_int32]
        L.ausaxs_gpu_server_usage.argtypes = [vp, i64, i64, i32]
        L.ausaxs_gpu_server_submit.argtypes = [vp, C.c_int32, C.c_int32, f64, f64, i64]
        L.ausaxs_gpu_server_poll.argtypes = [vp, C.c_int64, i32, f64, f64]
        L.ausaxs_gpu_server_wait.argtypes = [vp, C.c_int64, C.c_int32, f64, f64]
        L.ausaxs_gpu_server_completed.argtypes = [vp, i64, C.c_int32, i32]
        L.ausaxs_gpu_server_launch_count.argtypes = [vp, i64]
        L.ausaxs_gpu_server_body_center.argtypes = [vp, C.c_int32, C.c_int32, f64]
        L.ausaxs_gpu_server_coordinates.argtypes = [vp, C.c_int32, f32, f32]
        L.ausaxs_gpu_server_histogram.argtypes = [vp, C.c_int32, C.POINTER(HistResult)]
        L.ausaxs_gpu_hydrate.argtypes = [vp, f64, i32, C.c_int64, f64, f64, C.c_uint64, f64, C.c_int64, i64, i64, i32]
        L.ausaxs_hydrate_axes.argtypes = [f64, C.c_int64, f64]
        L.ausaxs_gpu_ctx_hydration_stats.argtypes = [vp, i64, i32]
        L.ausaxs_gpu_hydrate_device.argtypes = [vp, f64, i32, C.c_int64, f64, f64, C.c_uint64, f64, C.c_int64, i64, i64,
                                                i32]
        L.ausaxs_gpu_hydration_grid_create.argtypes = [vp, f64, C.POINTER(vp)]
        L.ausaxs_gpu_hydration_grid_destroy.argtypes = [vp]
        L.ausaxs_gpu_hydration_grid_add.argtypes = [vp, f64, i32, C.c_int64]
        L.ausaxs_gpu_hydration_grid_remove.argtypes = [vp, f64, i32, C.c_int64]
        L.ausaxs_gpu_hydration_grid_hydrate.argtypes = [vp, f64, i32, C.c_int64, f64, C.c_uint64, f64, C.c_int64, i64,
                                                        i64, i32]
        _lib = L
        return L


def smem_atomic_rate(device: int = 0, conflict_free: bool = True, wide: bool = False):
    """(shared-memory atomics per second over the device, kernel milliseconds); wide: 64-bit atomics."""
    r, ms = C.c_double(0.0), C.c_double(0.0)
    mode = int(bool(conflict_free)) | (2 if wide else 0)
    check(load().ausaxs_gpu_smem_atomic_rate(device, mode, C.byref(r), C.byref(ms)))
    return r.value, ms.value


def check(rc: int):
    if rc != OK:
        raise AusaxsError(rc, load().ausaxs_gpu_last_error().decode())


def fptr(a: np.ndarray | None, ctype=C.c_float):
    if a is None:
        return C.cast(0, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


def dptr(a: np.ndarray | None):
    return fptr(a, C.c_double)


def devptr(x, ctype=C.c_double):
    """Pointer of a device buffer (an integer address or anything with data_ptr())."""
    addr = x.data_ptr() if hasattr(x, "data_ptr") else int(x)
    return C.cast(C.c_void_p(addr), C.POINTER(ctype))


class Context:
    """One CUDA context handle of the library (its own stream and workspace)."""

    def __init__(self, device: int = 0):
        L = load()
        h = C.c_void_p()
        check(L.ausaxs_gpu_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None):
        check(load().ausaxs_gpu_ctx_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    @property
    def launches(self) -> int:
        return int(load().ausaxs_gpu_ctx_launch_count(self.h))

    def enable_timing(self, on: bool = True):
        check(load().ausaxs_gpu_ctx_enable_timing(self.h, int(on)))

    def fp64_columns(self) -> int:
        n = C.c_int32(0)
        check(load().ausaxs_gpu_ctx_fp64_columns(self.h, C.byref(n)))
        return n.value

    def tc_error_estimate(self, nq: int):
        out = np.zeros(nq)
        check(load().ausaxs_gpu_ctx_tc_error_estimate(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), nq))
        return out

    def kernel_time(self, cls: int):
        """(total ms, launches) of a kernel class: 0 pair histograms, 1 finalisation, 2 FP64 Debye,
        3 tensor-core Debye."""
        ms = C.c_double(0)
        n = C.c_int64(0)
        check(load().ausaxs_gpu_ctx_kernel_time(self.h, cls, C.byref(ms), C.byref(n)))
        return ms.value, n.value


def linear_lsq(ctx: "Context", data, model, err) -> np.ndarray:
    """{a, b, sigma_a, sigma_b, chi2} of model ~ a * data + b (fitter::detail::LinearLeastSquares::fit)."""
    data, model, err = (np.ascontiguousarray(x, np.float64) for x in (data, model, err))
    out = np.zeros(5)
    check(load().ausaxs_gpu_linear_lsq(ctx.h, dptr(data), dptr(model), dptr(err), len(data), dptr(out)))
    return out


_default = {}


EXV_FROM_GRID = -1


def grid_exv(ctx: "Context", atoms, waters):
    """Excluded-volume dummies of the molecular grid (RawGridExv) and the grid volume: ([n, 4] records, volume).
    One device pass when the first guess of the dummy count (40 per atom) suffices, else a second."""
    a = np.ascontiguousarray(atoms, np.float32).reshape(-1, 4)
    w = np.ascontiguousarray(waters, np.float32).reshape(-1, 4)
    n = C.c_int64(0)
    vol = C.c_double(0)
    cap = 40 * len(a) + 1024
    while True:
        out = np.zeros((cap, 4), np.float32)
        rc = load().ausaxs_gpu_grid_exv(ctx.h, fptr(a), len(a), fptr(w), len(w), 1, fptr(out), cap, C.byref(n),
                                        C.byref(vol))
        if rc == ERR_CAPACITY and n.value > cap:
            cap = n.value
            continue
        check(rc)
        return out[: n.value], vol.value


def grid_exv_device(ctx: "Context", atoms_dev, n_atoms: int, waters_dev, n_waters: int, out_dev, capacity: int):
    """The same on device records (device addresses); writes the dummies to out_dev.  Returns (count, volume)."""
    n = C.c_int64(0)
    vol = C.c_double(0)
    check(load().ausaxs_gpu_grid_exv(ctx.h, devptr(atoms_dev, C.c_float), n_atoms, devptr(waters_dev, C.c_float),
                                     n_waters, 0, devptr(out_dev, C.c_float), capacity, C.byref(n), C.byref(vol)))
    return n.value, vol.value


HYDRATE_DIRECTIONS = 26


def hydrate_axes(atoms) -> np.ndarray:
    """The axes Grid(bodies) builds around the atoms for the hydration: {min x, y, z, bins x, y, z}."""
    a = np.ascontiguousarray(np.asarray(atoms, np.float64).reshape(-1, 3))
    out = np.zeros(6)
    check(load().ausaxs_hydrate_axes(fptr(a, C.c_double), len(a), fptr(out, C.c_double)))
    return out


def _hydrate_inputs(atoms, ff_types, noise):
    a = np.ascontiguousarray(np.asarray(atoms, np.float64).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(ff_types, np.int32).reshape(-1))
    nz = None
    if noise is not None:
        nz = np.zeros((HYDRATE_DIRECTIONS * len(a), 3))
        src = np.asarray(noise, np.float64).reshape(-1, 3)[: len(nz)]
        nz[: len(src)] = src
    return a, f, nz


def _hydrate_call(fn, a, nz):
    """Runs fn(out, cap, n, cand, rounds) with a growing capacity; returns (waters, candidates, rounds)."""
    n = C.c_int64(0)
    rounds = C.c_int32(0)
    cap = max(1024, 2 * len(a))
    while True:
        out = np.zeros((cap, 3))
        cand = np.zeros(cap, np.int64)
        rc = fn(fptr(out, C.c_double), cap, C.byref(n), fptr(cand, C.c_int64), C.byref(rounds))
        if rc == ERR_CAPACITY and n.value > cap:
            cap = n.value
            continue
        check(rc)
        return out[: n.value], cand[: n.value], rounds.value


def hydration_stats(ctx: "Context"):
    """(candidates that passed the static tests, rounds) of the context's last hydration."""
    s, r = C.c_int64(0), C.c_int32(0)
    check(load().ausaxs_gpu_ctx_hydration_stats(ctx.h, C.byref(s), C.byref(r)))
    return s.value, r.value


def hydrate_device(ctx: "Context", atoms_dev, ff_dev, n_atoms: int, axes, out_dev, capacity: int, cand_dev=None,
                   noise_dev=None, seed: int = 0):
    """ausaxs_gpu_hydrate_device: device atoms (n x 3 double), types (int32), optional noise table;
    writes the waters (and candidate indices) into device buffers.  Returns (count, rounds)."""
    ax = np.ascontiguousarray(np.asarray(axes, np.float64)[:6])
    n = C.c_int64(0)
    rounds = C.c_int32(0)
    check(load().ausaxs_gpu_hydrate_device(
        ctx.h, devptr(atoms_dev, C.c_double), devptr(ff_dev, C.c_int32), n_atoms, fptr(ax, C.c_double),
        None if noise_dev is None else devptr(noise_dev, C.c_double), int(seed), devptr(out_dev, C.c_double), capacity,
        C.byref(n), None if cand_dev is None else devptr(cand_dev, C.c_int64), C.byref(rounds)))
    return n.value, rounds.value


class HydrationGrid:
    """A hydration grid kept on the device across calls (ausaxs_gpu_hydration_grid_*), as the reference
    keeps a molecule's grid::Grid between rigid-body steps: add(atoms, ff) = Grid::add with the volume
    expansion, remove(atoms, ff) = Grid::remove of atoms at those (current) coordinates, hydrate(atoms,
    ff, noise, seed) = RadialHydration over the grid's members in the order given."""

    def __init__(self, ctx: "Context", axes):
        self.ctx = ctx
        self.axes = np.ascontiguousarray(np.asarray(axes, np.float64)[:6])
        h = C.c_void_p()
        check(load().ausaxs_gpu_hydration_grid_create(ctx.h, fptr(self.axes, C.c_double), C.byref(h)))
        self.h = h

    def add(self, atoms, ff_types):
        a, f, _ = _hydrate_inputs(atoms, ff_types, None)
        check(load().ausaxs_gpu_hydration_grid_add(self.h, fptr(a, C.c_double), fptr(f, C.c_int32), len(a)))

    def remove(self, atoms, ff_types):
        a, f, _ = _hydrate_inputs(atoms, ff_types, None)
        check(load().ausaxs_gpu_hydration_grid_remove(self.h, fptr(a, C.c_double), fptr(f, C.c_int32), len(a)))

    def hydrate(self, atoms, ff_types, noise=None, seed: int = 0):
        a, f, nz = _hydrate_inputs(atoms, ff_types, noise)
        L = load()
        return _hydrate_call(lambda out, cap, n, cand, rounds: L.ausaxs_gpu_hydration_grid_hydrate(
            self.h, fptr(a, C.c_double), fptr(f, C.c_int32), len(a), fptr(nz, C.c_double), int(seed), out, cap, n,
            cand, rounds), a, nz)

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_hydration_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hydrate(ctx: "Context", atoms, ff_types, axes=None, noise=None, seed: int = 0):
    """RadialHydration on a fresh grid on the device (ausaxs_gpu_hydrate): waters [m, 3] (double) in the
    reference's order, their candidate indices (atom * 26 + direction) and the rounds the device
    took.  atoms in the order the generator visits them; noise: [n * 26, 3] displacements or None
    (then seed != 0 draws Gaussian ones of sigma 0.75 A on the device)."""
    a, f, nz = _hydrate_inputs(atoms, ff_types, noise)
    ax = None if axes is None else np.ascontiguousarray(np.asarray(axes, np.float64)[:6])
    L = load()
    return _hydrate_call(lambda out, cap, n, cand, rounds: L.ausaxs_gpu_hydrate(
        ctx.h, fptr(a, C.c_double), fptr(f, C.c_int32), len(a), fptr(ax, C.c_double), fptr(nz, C.c_double),
        int(seed), out, cap, n, cand, rounds), a, nz)


class Calculator:
    """hist::distance_calculator::SimpleCalculator<true, vbw> on the device (ausaxs_gpu_calculator_*):
    enqueue_calculate_self / enqueue_calculate_cross with scaling factors and merge ids, then run()
    -> {"self": {id: (value, count, distance_sum)}, "cross": {...}}, each bin_count long."""

    def __init__(self, ctx: Context, bin_width: float = 0.25, bin_count: int = 8000):
        self.ctx = ctx
        self.bin_count = bin_count
        self._keep = []  # the arrays must stay valid until run()
        h = C.c_void_p()
        check(load().ausaxs_gpu_calculator_create(ctx.h, float(bin_width), int(bin_count), C.byref(h)))
        self.h = h

    def _pts(self, p):
        a = np.ascontiguousarray(p, np.float32).reshape(-1, 4)
        self._keep.append(a)
        return a

    def enqueue_calculate_self(self, points, scaling: int = 1, merge_id: int = -1) -> int:
        a = self._pts(points)
        r = C.c_int32(0)
        check(load().ausaxs_gpu_calculator_enqueue_self(self.h, fptr(a), len(a), int(scaling), int(merge_id), C.byref(r)))
        return r.value

    def enqueue_calculate_cross(self, points_1, points_2, scaling: int = 1, merge_id: int = -1) -> int:
        a, b = self._pts(points_1), self._pts(points_2)
        r = C.c_int32(0)
        check(load().ausaxs_gpu_calculator_enqueue_cross(self.h, fptr(a), len(a), fptr(b), len(b), int(scaling),
                                                        int(merge_id), C.byref(r)))
        return r.value

    def run(self) -> dict:
        L = load()
        ns, nc = C.c_int32(0), C.c_int32(0)
        check(L.ausaxs_gpu_calculator_run(self.h, C.byref(ns), C.byref(nc)))
        self._keep = []
        out = {"self": {}, "cross": {}}
        for cross, key, n in ((0, "self", ns.value), (1, "cross", nc.value)):
            ids = np.zeros(max(1, n), np.int32)
            m = C.c_int32(0)
            check(L.ausaxs_gpu_calculator_result_ids(self.h, cross, ids.ctypes.data_as(C.POINTER(C.c_int32)), n,
                                                     C.byref(m)))
            for i in ids[:m.value]:
                v, c, d = (np.zeros(self.bin_count) for _ in range(3))
                check(L.ausaxs_gpu_calculator_result(self.h, cross, int(i), dptr(v), dptr(c), dptr(d)))
                out[key][int(i)] = (v, c, d)
        return out

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_calculator_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device: int = 0) -> Context:
    if device not in _default:
        _default[device] = Context(device)
    return _default[device]


class Structure:
    """A device-resident structure (ausaxs_gpu_structure_*): upload once, profile many times."""

    def __init__(self, ctx: Context, atoms, waters, exv=None, ff_typed: bool = True, exv_from_grid: bool = False):
        """exv: excluded-volume dummy records, or exv_from_grid: the dummies of the molecular grid."""
        self.ctx = ctx
        self._a = np.ascontiguousarray(atoms, np.float32)
        self._w = np.ascontiguousarray(waters, np.float32)
        self._x = None if exv is None else np.ascontiguousarray(exv, np.float32)
        nx = EXV_FROM_GRID if exv_from_grid else (0 if self._x is None else len(self._x))
        h = C.c_void_p()
        check(load().ausaxs_gpu_structure_create(ctx.h, int(ff_typed), fptr(self._a), len(self._a), fptr(self._w),
                                                 len(self._w), fptr(self._x), nx, 1, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_structure_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def profile_device(self, cfg: HistConfig, q_dev, nq: int, params: DebyeParams, I_dev, prof_dev=None):
        """Enqueue coordinates -> I(q) on the context's stream; q/I/profiles are device addresses."""
        check(load().ausaxs_gpu_structure_profile(self.ctx.h, self.h, C.byref(cfg), devptr(q_dev), nq,
                                                  C.byref(params), devptr(I_dev),
                                                  devptr(prof_dev) if prof_dev is not None else C.cast(0, C.POINTER(C.c_double))))

    def fit_device(self, cfg: HistConfig, q_dev, y_dev, sigma_dev, n: int, base: DebyeParams, options: FitOptions,
                   I_fit_dev=None) -> FitResult:
        """ausaxs_gpu_structure_fit: q, data, errors (and the fitted curve) are device addresses."""
        out = FitResult()
        check(load().ausaxs_gpu_structure_fit(self.ctx.h, self.h, C.byref(cfg), devptr(q_dev), devptr(y_dev),
                                              devptr(sigma_dev), n, C.byref(base), C.byref(options), C.byref(out),
                                              devptr(I_fit_dev) if I_fit_dev is not None else C.cast(0, C.POINTER(C.c_double))))
        return out

    def histogram(self, cfg: HistConfig, bin_count: int):
        ff = cfg.manager != MANAGER_MT
        bufs = {k: np.zeros(n) for k, n in [("aa", (225 if ff else 1) * bin_count), ("aw", (15 if ff else 1) * bin_count),
                                             ("ww", bin_count), ("tot", bin_count), ("d_axis", bin_count),
                                             ("d_axis_ax", bin_count), ("d_axis_xx", bin_count)]}
        r = HistResult()
        for k, v in bufs.items():
            setattr(r, k, dptr(v))
        check(load().ausaxs_gpu_structure_histogram(self.ctx.h, self.h, C.byref(cfg), C.byref(r)))
        return r, bufs


class Batch:
    """Many device-resident structures profiled together (ausaxs_gpu_batch_*)."""

    def __init__(self, ctx: Context, cfg: HistConfig, atoms: list, waters: list, exv: list | None = None,
                 z_exv=None):
        self.ctx = ctx
        self.cfg = cfg
        self.n = len(atoms)

        def cat(parts):
            parts = [np.ascontiguousarray(p, np.float32).reshape(-1, 4) for p in parts]
            off = np.zeros(len(parts) + 1, np.int64)
            off[1:] = np.cumsum([len(p) for p in parts])
            data = np.ascontiguousarray(np.concatenate(parts) if off[-1] else np.zeros((1, 4), np.float32))
            return data, off

        self._a, self._ao = cat(atoms)
        self._w, self._wo = cat(waters)
        self._x, self._xo = (None, None) if exv is None else cat(exv)
        self._z = None if z_exv is None else np.ascontiguousarray(z_exv, np.float64)
        i64 = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_int64))
        h = C.c_void_p()
        check(load().ausaxs_gpu_batch_create(ctx.h, C.byref(cfg), self.n, fptr(self._a), i64(self._ao), fptr(self._w),
                                             i64(self._wo), fptr(self._x), i64(self._xo), dptr(self._z), 1, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self):
        """(chosen candidate, per-candidate milliseconds of the pair launches)."""
        times = np.zeros(16)
        c = C.c_int32(-1)
        check(load().ausaxs_gpu_batch_autotune(self.h, C.byref(c), dptr(times), len(times)))
        return c.value, times

    @staticmethod
    def candidate(index: int) -> dict:
        v = [C.c_int32() for _ in range(4)]
        check(load().ausaxs_gpu_batch_candidate(index, *[C.byref(x) for x in v]))
        return dict(zip(("tile_small", "tile_large", "threshold", "by_class"), [x.value for x in v]))

    def profile(self, q, params: DebyeParams) -> np.ndarray:
        q = np.ascontiguousarray(q, np.float64)
        out = np.zeros(self.n * len(q))
        check(load().ausaxs_gpu_batch_profile(self.h, dptr(q), len(q), C.byref(params), dptr(out)))
        return out.reshape(self.n, len(q))

    def profile_device(self, q_dev, nq: int, params: DebyeParams, I_dev):
        check(load().ausaxs_gpu_batch_profile_device(self.h, devptr(q_dev), nq, C.byref(params), devptr(I_dev)))

    def fp64_columns(self) -> int:
        """(structure, q) values of the last profile recomputed in FP64 (waits for it)."""
        n = C.c_int64(0)
        check(load().ausaxs_gpu_batch_fp64_columns(self.h, C.byref(n)))
        return n.value

    def pair_time(self) -> float:
        """Device milliseconds of the last profile's pair stage (waits for it)."""
        ms = C.c_double(0.0)
        check(load().ausaxs_gpu_batch_pair_time(self.h, C.byref(ms)))
        return ms.value

    def set_points(self, atoms: list, waters: list, z_exv=None):
        """New coordinates for every structure (same shapes and atom types as at creation) and, when
        given, new excluded-volume charges; the next profile replays the captured graph on them."""
        a = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 4) for p in atoms])
                                 if self._ao[-1] else np.zeros((1, 4), np.float32))
        w = np.ascontiguousarray(np.concatenate([np.asarray(p, np.float32).reshape(-1, 4) for p in waters])
                                 if self._wo[-1] else np.zeros((1, 4), np.float32))
        if self._ao[-1] and a.shape != self._a.shape or self._wo[-1] and w.shape != self._w.shape:
            raise AusaxsError(ERR_ARGUMENT, "set_points needs the creation shapes")
        z = None if z_exv is None else np.ascontiguousarray(z_exv, np.float64)
        if z is not None and z.shape != (self.n,):
            raise AusaxsError(ERR_ARGUMENT, "z_exv needs one value per structure")
        check(load().ausaxs_gpu_batch_set_points(self.h, fptr(a), fptr(w), dptr(z), 1))

    def set_points_device(self, atoms_dev, waters_dev, z_exv=None):
        """As set_points from device tensors in the creation layout (float32 [rows, 4]); asynchronous."""
        z = None if z_exv is None else np.ascontiguousarray(z_exv, np.float64)
        check(load().ausaxs_gpu_batch_set_points(self.h, devptr(atoms_dev, C.c_float), devptr(waters_dev, C.c_float),
                                                 dptr(z), 0))

    def histogram(self, index: int, bin_count: int):
        bufs = {k: np.zeros(n) for k, n in [("aa", 225 * bin_count), ("aw", 15 * bin_count), ("ww", bin_count),
                                             ("tot", bin_count), ("d_axis", bin_count), ("d_axis_ax", bin_count),
                                             ("d_axis_xx", bin_count)]}
        r = HistResult()
        for k, v in bufs.items():
            setattr(r, k, dptr(v))
        check(load().ausaxs_gpu_batch_histogram(self.h, index, C.byref(r)))
        return r, bufs



class Server:
    """Rigid-body serving (ausaxs_gpu_server_*): device-resident multi-body assemblies, one body moved
    per request, I(q) and the linear fit against a target returned per request."""

    def __init__(self, device: int = 0, hbm_budget: int = 8 << 30, max_inflight: int = 64, slots_per_assembly: int = 4):
        h = C.c_void_p()
        check(load().ausaxs_gpu_server_create(device, int(hbm_budget), max_inflight, slots_per_assembly, C.byref(h)))
        self.h = h
        self.nq = {}
        self.n_atoms = {}
        self.n_waters = {}

    def set_policy(self, policy: int):
        """0: concurrent per-assembly streams with small moves at high priority; k > 0: submission order
        over k streams (at most k moves share the device)."""
        check(load().ausaxs_gpu_server_set_policy(self.h, int(policy)))

    def close(self):
        if getattr(self, "h", None):
            load().ausaxs_gpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, cfg: HistConfig, bodies_atoms: list, bodies_waters: list, q, params: DebyeParams,
              target=None, target_err=None, margin: float = 20.0):
        """bodies_atoms[k]: [n_k, 4] {x, y, z, ff}; bodies_waters[k]: [m_k, 4] {x, y, z, w}.  Returns (id, footprint)."""
        def cat(parts):
            parts = [np.ascontiguousarray(p, np.float32).reshape(-1, 4) for p in parts]
            off = np.zeros(len(parts) + 1, np.int64)
            off[1:] = np.cumsum([len(p) for p in parts])
            return np.ascontiguousarray(np.concatenate(parts) if off[-1] else np.zeros((1, 4), np.float32)), off

        a, ao = cat(bodies_atoms)
        w, wo = cat(bodies_waters)
        q = np.ascontiguousarray(q, np.float64)
        tg = None if target is None else np.ascontiguousarray(target, np.float64)
        te = None if target_err is None else np.ascontiguousarray(target_err, np.float64)
        i = C.c_int32(-1)
        fp = C.c_int64(0)
        i64 = lambda x: x.ctypes.data_as(C.POINTER(C.c_int64))
        rc = load().ausaxs_gpu_server_admit(self.h, C.byref(cfg), len(bodies_atoms), fptr(a), i64(ao), fptr(w), i64(wo),
                                            float(margin), dptr(q), len(q), C.byref(params), dptr(tg), dptr(te),
                                            C.byref(i), C.byref(fp))
        check(rc)
        self.nq[i.value] = len(q)
        self.n_atoms[i.value] = int(ao[-1])
        self.n_waters[i.value] = int(wo[-1])
        return i.value, fp.value

    def release(self, id: int):
        check(load().ausaxs_gpu_server_release(self.h, id))

    def usage(self):
        u, b, n = C.c_int64(), C.c_int64(), C.c_int32()
        check(load().ausaxs_gpu_server_usage(self.h, C.byref(u), C.byref(b), C.byref(n)))
        return u.value, b.value, n.value

    def submit(self, id: int, body: int = -1, R=None, t=None) -> int:
        Rm = None if R is None else np.ascontiguousarray(R, np.float64).reshape(9)
        tv = None if t is None else np.ascontiguousarray(t, np.float64).reshape(3)
        tk = C.c_int64(-1)
        check(load().ausaxs_gpu_server_submit(self.h, id, body, dptr(Rm), dptr(tv), C.byref(tk)))
        return tk.value

    def try_submit(self, id: int, body: int = -1, R=None, t=None):
        """Ticket, or None when no slot is free."""
        try:
            return self.submit(id, body, R, t)
        except AusaxsError as e:
            if e.code == ERR_CAPACITY:
                return None
            raise

    def poll(self, ticket: int, id: int):
        I = np.zeros(self.nq[id])
        fit = np.zeros(5)
        done = C.c_int32(0)
        check(load().ausaxs_gpu_server_poll(self.h, ticket, C.byref(done), dptr(I), dptr(fit)))
        return (I, fit) if done.value else None

    def wait(self, ticket: int, id: int, timeout_ms: int = 10000):
        I = np.zeros(self.nq[id])
        fit = np.zeros(5)
        check(load().ausaxs_gpu_server_wait(self.h, ticket, timeout_ms, dptr(I), dptr(fit)))
        return I, fit

    def completed(self, capacity: int = 256):
        """Tickets whose results are ready (collect them with poll)."""
        out = np.zeros(capacity, np.int64)
        n = C.c_int32(0)
        check(load().ausaxs_gpu_server_completed(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)), capacity,
                                                 C.byref(n)))
        return out[: n.value].tolist()

    def launches(self) -> int:
        n = C.c_int64(0)
        check(load().ausaxs_gpu_server_launch_count(self.h, C.byref(n)))
        return n.value

    def body_center(self, id: int, body: int) -> np.ndarray:
        c = np.zeros(3)
        check(load().ausaxs_gpu_server_body_center(self.h, id, body, dptr(c)))
        return c

    def coordinates(self, id: int):
        a = np.zeros((max(1, self.n_atoms[id]), 4), np.float32)
        w = np.zeros((max(1, self.n_waters[id]), 4), np.float32)
        check(load().ausaxs_gpu_server_coordinates(self.h, id, fptr(a), fptr(w)))
        return a[: self.n_atoms[id]], w[: self.n_waters[id]]

    def histogram(self, id: int, bin_count: int):
        bufs = {k: np.zeros(n) for k, n in [("aa", 225 * bin_count), ("aw", 15 * bin_count), ("ww", bin_count),
                                             ("tot", bin_count), ("d_axis", bin_count), ("d_axis_ax", bin_count),
                                             ("d_axis_xx", bin_count)]}
        r = HistResult()
        for k, v in bufs.items():
            setattr(r, k, dptr(v))
        check(load().ausaxs_gpu_server_histogram(self.h, id, C.byref(r)))
        m = r.max_bin
        return {"max_bin": m, "aa": bufs["aa"][: 225 * m].reshape(15, 15, m), "aw": bufs["aw"][: 15 * m].reshape(15, m),
                "ww": bufs["ww"][:m], "d_axis": bufs["d_axis"][:m]}
