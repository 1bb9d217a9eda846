"""Benchmark of the Debye hot path: I(q) profiles per second on a B200.

Default workload (single GPU): the batched configuration -- 256 independent globules, atom counts
log-uniform in [500, 50,000], waters 20 % of the atoms, 0.25 A bins, 400 q in [0.005, 0.8],
HistogramManagerMTFFAvg semantics, generated from a seed (no dataset).  One step = every
structure's coordinates -> pair histograms -> FP64 Debye transform -> I(q), one CUDA-graph replay.

  value            : batched profiles/s, structures resident in HBM
  plain_sequential : the same 256 profiles as 256 plain single-structure calls, and the ratio
  e2e              : profiles/s through the C ABI from pinned host buffers (the batch created,
                     profiled and destroyed every step: H2D of all points, D2H of every I(q))
  roofline         : the pair kernel against min(FP32 bound, measured shared-atomic bound)
  serving          : the rigid-body serving configuration (64 chains of 8-body assemblies): moves/s
                     at saturation, p50/p99 latency at 25/50/75 % of it, lone-request latencies

Other workloads (--workload): cfg0, cfg1 (50k-atom FFGrid, 1,000 q), cfg2 (500k-atom shell), cfg4
(serving alone), gridexv, hydrate, fit, symmetry, atomics-peak.
Under torchrun (N > 1) every rank runs its own replica (weak scaling).
``--impl reference`` times the reference implementation compiled from its sources (oracle/_ref)
on the host cores: for the default workload, whole structures of the batch in size-stratified
chunks, one chunk per step, so the timed steps cover the batch once (no extrapolation).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# warp instructions per 32 pair evaluations of the pair kernel at 0.25 A bins (the batch and serving
# configurations; the bin rounding fused with the power-of-two inverse width), counted by ncu on the
# batch's pair launches (smsp__inst_executed / (shared atomics / 2),
# profiles/pairhist_kernel_batch_64_structures.md)
INSTR_PER_PAIR = 31.1
# DRAM bytes (read + write) of the pair launches of one step of the 256-structure batch: 16.6 MB per pass
# measured by ncu on its first 64 structures (0.86M points), scaled by points to the batch's 3.66M
BATCH_PAIR_TRAFFIC_BYTES = 7.0e7
METRIC = "I(q) profiles/s & p99 latency vs plain GPU path at ≤1e-4 rel. I(q) error"
UNIT = "profiles/s"


def max_over_ranks(x: float, world: int) -> float:
    """The largest value of x over all ranks (a time: the job is as slow as its slowest rank)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def workload(name: str, subunit: int = 0, atoms: int = 0, structures: int = 0):
    """subunit (cfg2 only): atoms per icosahedral subunit; smaller shells keep the radius and bin count
    of the full shell.  atoms (cfg1 only): a globule of the same composition and density.  structures
    (cfg3 only): the first structures of the seeded batch.  All three are profiling cases."""
    from ausaxs_b200 import synth

    if name == "cfg2" and subunit:
        return synth.cfg2(subunit=subunit)
    if name == "cfg1" and atoms:
        return synth.cfg1(atoms=atoms)
    if name == "cfg3" and structures:
        return synth.cfg3(count=structures)
    return {"cfg0": synth.cfg0, "cfg1": synth.cfg1, "cfg2": synth.cfg2, "cfg3": synth.cfg3}[name]()


def pair_count(m, grid: bool) -> int:
    na, nw = m.size_atom(), m.size_water()
    nx = len(m.exv) if (grid and m.exv is not None) else 0
    return na * (na - 1) // 2 + na * nw + nw * (nw - 1) // 2 + (na * nx + nw * nx + nx * (nx - 1) // 2 if grid else 0)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        import tempfile

        self.path = os.path.join(tempfile.gettempdir(), f"ausaxs_b200_clocks_{os.getpid()}_{id(self)}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
            self.text = open(self.path).read() if os.path.exists(self.path) else ""
            try:
                os.remove(self.path)
            except OSError:
                pass

    def summary(self):
        text = getattr(self, "text", "")
        if not self.proc or not text:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in text.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def reference_sample(m, grid: bool, target_pairs: float, seed: int = 5):
    """A uniform subsample of every point set with about target_pairs pairs."""
    full = pair_count(m, grid)
    f = min(1.0, (target_pairs / max(full, 1)) ** 0.5)
    rng = np.random.default_rng(seed)

    def pick(a):
        if a is None or len(a) == 0:
            return a
        k = max(1, int(round(len(a) * f)))
        return np.sort(rng.choice(len(a), k, replace=False))

    ia, iw = pick(m.atoms), pick(m.waters)
    ix = pick(m.exv) if grid else None
    from ausaxs_b200.hist import Molecule

    s = Molecule(atoms=m.atoms[ia], ff_types=m.ff_types[ia], weights=m.weights[ia], waters=m.waters[iw],
                 water_weights=m.water_weights[iw], exv=(m.exv[ix] if grid else None),
                 volume=m.volume * len(ia) / len(m.atoms))
    return s, pair_count(s, grid) / full


def time_reference(m, wl, steps: int, warmup: int, target_pairs: float = 4e9):
    """The reference (compiled from source) on a bounded sample; returns (profiles/s, details)."""
    from oracle import py as O

    if not O.ref_available():
        return None, {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    grid = wl.manager == "ffgrid"
    threads = max(1, (os.cpu_count() or 2) - 1)
    O.ref(threads)
    O.ref_set_axes(wl.bin_width, 8000, 1e-4, 1.0)
    O.ref_set_simple_exv(False)
    s, frac = reference_sample(m, grid, target_pairs)
    rm = O.RefMolecule(s.atoms, s.weights, s.ff_types, s.waters, s.water_weights, volume=s.volume)
    rm.set_manager(wl.manager, exv_xyz=s.exv if grid else None)
    times = []
    for it in range(warmup + steps):
        h = rm.calculate()
        _, _, _, t_debye = h.debye()
        # the reference's transform runs on its fixed 200-point axis; scale to this workload's q count
        t = h.seconds / frac + t_debye * (len(wl.q) / 200.0)
        if it >= warmup:
            times.append(t)
    per = statistics.median(times)
    detail = {"cores": threads, "sample": (f"uniform subsample of atoms/waters/exv with {frac:.4f} of the pairs "
                                           f"({s.size_atom()} atoms, {s.size_water()} waters, "
                                           f"{0 if s.exv is None else len(s.exv)} exv); calculate_all() time scaled by "
                                           f"pairs, debye_transform() time scaled by q count"),
              "kind": "reference"}
    return 1.0 / per, detail


def moved_pose(batch, seed: int, shrink: float = 0.98):
    """Another pose of every structure of a batch, in its creation layout: atoms and waters rotated
    about the atoms' centroid and shrunk by `shrink` (pair distances only shorten, so the bins planned
    at creation hold them), form-factor types kept; excluded-volume charges follow the volume."""
    rng = np.random.default_rng(seed)
    a, w = batch._a.copy(), batch._w.copy()
    for i in range(batch.n):
        a0, a1, w0, w1 = batch._ao[i], batch._ao[i + 1], batch._wo[i], batch._wo[i + 1]
        r, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        c = a[a0:a1, :3].astype(np.float64).mean(axis=0) if a1 > a0 else np.zeros(3)
        for lo, hi, arr in ((a0, a1, a), (w0, w1, w)):
            if hi > lo:
                arr[lo:hi, :3] = (((arr[lo:hi, :3] - c) @ r.T) * shrink + c).astype(np.float32)
    z = np.ascontiguousarray(batch._z * shrink ** 3)
    return a, w, z


def batch_chunks(wl, n_chunks: int):
    """Size-stratified partition of a batch's structures into n_chunks chunks (structures ranked by
    pair count, dealt round-robin), so that every chunk has the batch's size mix and the chunks
    together are the whole batch."""
    ranked = sorted(range(len(wl.molecules)), key=lambda i: -pair_count(wl.molecules[i], False))
    n_chunks = max(1, min(n_chunks, len(ranked)))
    return [ranked[c::n_chunks] for c in range(n_chunks)]


def time_reference_structures(wl, picked, O):
    """Seconds of the reference for the structures `picked`: calculate_all() + debye_transform() each.
    The reference's FF-typed transform runs on its fixed 200-point q axis; its time is scaled to the
    workload's q count (the transform is < 2 % of a structure's time)."""
    t = 0.0
    for i in picked:
        m = wl.molecules[i]
        rm = O.RefMolecule(m.atoms, m.weights, m.ff_types, m.waters, m.water_weights, volume=m.volume)
        rm.set_manager(wl.manager)
        h = rm.calculate()
        _, _, _, t_debye = h.debye()
        t += h.seconds + t_debye * (len(wl.q) / 200.0)
    return t


def time_reference_batch(wl, steps: int, warmup: int, n_chunks: int = 0):
    """The reference over the batch in size-stratified chunks of whole structures: step k runs chunk
    k mod n_chunks (n_chunks = steps by default, so the timed steps cover every structure once).
    Returns (profiles/s = structures timed / seconds, details); nothing is extrapolated."""
    from oracle import py as O

    if not O.ref_available():
        return None, {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    threads = max(1, (os.cpu_count() or 2) - 1)
    O.ref(threads)
    O.ref_set_axes(wl.bin_width, 8000, 1e-4, 1.0)
    O.ref_set_simple_exv(False)
    chunks = batch_chunks(wl, n_chunks or steps)
    done, secs = 0, 0.0
    for it in range(warmup + steps):
        c = chunks[(it - warmup) % len(chunks)] if it >= warmup else chunks[(len(chunks) - 1 - it) % len(chunks)]
        t = time_reference_structures(wl, c, O)
        if it >= warmup:
            done += len(c)
            secs += t
    covered = min(steps, len(chunks)) / len(chunks)
    detail = {"cores": threads, "kind": "reference",
              "sample": (f"{done} structures of the {len(wl.molecules)} in {steps} size-stratified chunks "
                         f"({covered:.3f} of the batch; each structure: calculate_all() + debye_transform(), the "
                         f"transform's 200-q time scaled to {len(wl.q)} q); no pair-count extrapolation"),
              "seconds": secs}
    return done / secs, detail


def batch_config(wl):
    """The workload's identity, printed unchanged by both arms."""
    mols = wl.molecules
    return {"workload": wl.name, "structures": len(mols), "atoms_total": int(sum(m.size_atom() for m in mols)),
            "waters_total": int(sum(m.size_water() for m in mols)),
            "pairs_per_step": int(sum(pair_count(m, False) for m in mols)), "bin_width": wl.bin_width,
            "q_points": len(wl.q), "q_range": [float(wl.q[0]), float(wl.q[-1])], "manager": wl.manager,
            "seed": 31}


def pair_roofline(pairs_per_launch: float, kernel_ms: float, sm_mhz: float, sms: int, atomic_rate: float,
                  atomics_per_pair: int, instr_per_pair: float):
    """Roofline of the pair kernel as pair evaluations per second: the lower of the FP32 bound
    (sms x 128 lanes x f_SM / 9 FP32 operations per pair) and the shared-atomic bound (measured
    conflict-free atomics/s / atomics per pair).  A secondary figure compares against the issue rate
    at the kernel's own instruction count (ncu)."""
    achieved = pairs_per_launch / (kernel_ms / 1e3)
    fp32 = sms * 128 * sm_mhz * 1e6 / 9.0
    atom = atomic_rate / atomics_per_pair
    peak = min(fp32, atom)
    issue = sms * 4 * sm_mhz * 1e6 * 32 / instr_per_pair
    return {"bound": "fp32" if fp32 <= atom else "smem_atomic", "kernel": "pairhist_kernel",
            "achieved": achieved / 1e9, "peak": peak / 1e9, "unit": "Gpair/s", "frac": achieved / peak,
            "fp32_bound": fp32 / 1e9, "smem_atomic_bound": atom / 1e9, "smem_atomics_per_s": atomic_rate,
            "atomics_per_pair": atomics_per_pair, "sm_mhz": sm_mhz, "issue_frac": achieved / issue,
            "instr_per_pair": instr_per_pair, "kernel_ms_per_step": kernel_ms,
            "peak_source": (f"min({sms} SMs x 128 x {sm_mhz:.0f} MHz / 9 FP32 ops per pair, measured conflict-free "
                            f"shared atomics / {atomics_per_pair} per pair)")}


def run_batch(args, rank, world, local_rank):
    """Batched profiles of many structures (one graph replay per step) against one plain
    single-structure call per structure."""
    import ctypes as C

    import torch

    from ausaxs_b200 import _capi, hist

    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    stream = torch.cuda.Stream(local_rank)
    ctx = _capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    wl = workload(args.workload, structures=args.structures)
    mols = wl.molecules
    n = len(mols)
    nq = len(wl.q)
    pairs = sum(pair_count(m, False) for m in mols)
    # the exact-accumulation tensor-core transform (precision 2) with FP64 wherever its bound exceeds
    # the metric's 1e-4; the FP64 transform of the same histograms checks it after the timed steps
    params = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, args.precision, args.tolerance)
    params64 = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    B = hist.BatchedProfiles(mols, bin_width=wl.bin_width, bin_count=wl.bin_count, ctx=ctx)
    choice, cand_ms = B.autotune()
    q_dev = torch.tensor(wl.q, dtype=torch.float64, device=dev)
    I_dev = torch.zeros(n * nq, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    atomic_rate, _ = _capi.smem_atomic_rate(local_rank, True)
    atomic_rate_random, _ = _capi.smem_atomic_rate(local_rank, False)

    def step():
        B._b.profile_device(q_dev, nq, params, I_dev)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
            flush.fill_(1.0)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        launches0 = ctx.launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        pair_ms = []
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                step()
                ends[k].record(stream)
                flush.fill_(float(k))
                try:
                    pair_ms.append(B._b.pair_time())  # events inside the graph, read after the step ends
                except _capi.AusaxsError:
                    pair_ms.append(None)
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = sum(step_ms)
    total_ms = max_over_ranks(total_ms, world)
    value = world * n * args.steps / (total_ms / 1e3)
    I_batch = I_dev.cpu().numpy().reshape(n, nq)
    fp64_cols = B._b.fp64_columns()
    I64_dev = torch.zeros(n * nq, dtype=torch.float64, device=dev)
    with torch.cuda.stream(stream):
        B._b.profile_device(q_dev, nq, params64, I64_dev)
        torch.cuda.synchronize()
    I_fp64 = I64_dev.cpu().numpy().reshape(n, nq)
    tc_diff = float(np.max(np.abs(I_batch / I_fp64 - 1)))

    # the plain path: one resident structure per call, called n times in sequence on the same stream
    cfgs = []
    sts = []
    for m in mols:
        mgr = hist.HistogramManagerMTFFAvg(m, True, wl.bin_width, wl.bin_count, ctx)
        a, w, _ = mgr._inputs()
        cfgs.append(mgr.config())
        sts.append(_capi.Structure(ctx, a, w, None, ff_typed=True))
    I_plain = torch.zeros(n * nq, dtype=torch.float64, device=dev)

    def plain_pass():
        for i in range(n):
            sts[i].profile_device(cfgs[i], q_dev, nq, params, I_plain[i * nq:])

    with torch.cuda.stream(stream):
        plain_pass()
        torch.cuda.synchronize()
        plain_ms = []
        for k in range(max(1, min(3, args.steps))):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plain_pass()
            e1.record(stream)
            torch.cuda.synchronize()
            plain_ms.append(e0.elapsed_time(e1))
            flush.fill_(float(k))
    plain_value = n / (statistics.median(plain_ms) / 1e3)
    plain_diff = float(np.max(np.abs(I_plain.cpu().numpy().reshape(n, nq) / I_batch - 1)))
    for st in sts:
        st.close()

    # end to end through the C ABI from pinned host buffers (the compact records the caller holds).
    # The batch made above stays (plans, job tables, captured graph); every step uploads new
    # coordinates for all structures (two poses of each molecule, alternating: a rotation about the
    # centroid with a 2 % shrink, so the bins planned at creation still hold them) and new
    # excluded-volume charges, replays the graph and reads every I(q) back.
    L = _capi.load()
    poses = [(B._b._a, B._b._w, np.ascontiguousarray(B._b._z)), moved_pose(B._b, seed=11)]
    pins = [(torch.from_numpy(a).pin_memory(), torch.from_numpy(w).pin_memory(), z) for a, w, z in poses]
    pin_q = torch.from_numpy(np.ascontiguousarray(wl.q)).pin_memory()
    pin_I = torch.zeros(n * nq, dtype=torch.float64).pin_memory()
    h2d = int(pins[0][0].numel() * 4 + pins[0][1].numel() * 4 + n * 8 + nq * 8)
    d2h = int(n * nq * 8 + 8 + 16)  # every I(q); the rejection count; overflow and rejection flags

    def e2e_step(k):
        a, w, z = pins[k % 2]
        _capi.check(L.ausaxs_gpu_batch_set_points(B._b.h, _capi.devptr(a, C.c_float), _capi.devptr(w, C.c_float),
                                                  _capi.dptr(z), 1))
        _capi.check(L.ausaxs_gpu_batch_profile(B._b.h, _capi.devptr(pin_q), nq, C.byref(params),
                                               _capi.devptr(pin_I)))

    with torch.cuda.stream(stream):
        for k in range(max(2, args.warmup)):
            e2e_step(k)
        lat = []
        for k in range(args.steps):
            t0 = time.perf_counter()
            e2e_step(k)
            lat.append(time.perf_counter() - t0)
        Ie = pin_I.numpy().reshape(n, nq).copy()  # pose (steps - 1) % 2
    e2e = world * n * len(lat) / max_over_ranks(sum(lat), world)
    last = (args.steps - 1) % 2
    if last == 0:
        e2e_diff = float(np.max(np.abs(Ie / I_batch - 1)))
    else:  # the moved pose against a batch created from it
        a1, w1, z1 = poses[1]
        i64 = lambda x: x.ctypes.data_as(C.POINTER(C.c_int64))
        hb = C.c_void_p()
        _capi.check(L.ausaxs_gpu_batch_create(ctx.h, C.byref(B.cfg), n, _capi.fptr(a1), i64(B._b._ao),
                                              _capi.fptr(w1), i64(B._b._wo), None, None, _capi.dptr(z1), 1,
                                              C.byref(hb)))
        If = np.zeros(n * nq)
        _capi.check(L.ausaxs_gpu_batch_profile(hb, _capi.dptr(np.ascontiguousarray(wl.q)), nq, C.byref(params),
                                               _capi.dptr(If)))
        _capi.check(L.ausaxs_gpu_batch_destroy(hb))
        e2e_diff = float(np.max(np.abs(Ie / If.reshape(n, nq) - 1)))

    # a batch of structures not seen before: created (H2D, census, plans), profiled, read back and
    # destroyed per call
    zv = np.ascontiguousarray(B._b._z)
    i64 = lambda x: x.ctypes.data_as(C.POINTER(C.c_int64))
    lat_new = []
    for k in range(1 + min(3, args.steps)):
        t0 = time.perf_counter()
        hb = C.c_void_p()
        _capi.check(L.ausaxs_gpu_batch_create(ctx.h, C.byref(B.cfg), n, _capi.devptr(pins[0][0], C.c_float),
                                              i64(B._b._ao), _capi.devptr(pins[0][1], C.c_float), i64(B._b._wo),
                                              None, None, _capi.dptr(zv), 1, C.byref(hb)))
        _capi.check(L.ausaxs_gpu_batch_profile(hb, _capi.devptr(pin_q), nq, C.byref(params), _capi.devptr(pin_I)))
        _capi.check(L.ausaxs_gpu_batch_destroy(hb))
        if k:
            lat_new.append(time.perf_counter() - t0)
    e2e_new = world * n * len(lat_new) / max_over_ranks(sum(lat_new), world)

    peaks, peak_kind = load_peaks()
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    timed_pairs = [x for x in pair_ms if x is not None]
    kernel_ms = statistics.mean(timed_pairs) if timed_pairs else float(cand_ms[choice])
    roof = pair_roofline(pairs, kernel_ms, sm_mhz, sms, atomic_rate, 2, INSTR_PER_PAIR)
    if not timed_pairs:
        roof["kernel_ms_source"] = "autotuner's timing of the chosen pair plan (graph events unavailable)"
    roof["traffic"] = BATCH_PAIR_TRAFFIC_BYTES
    roof["smem_atomics_per_s_random_bins"] = atomic_rate_random
    roof["note"] = ("kernel_ms = device time of the pair stage (accumulator clearing + every pair launch of the "
                    "graph), events inside the graph, mean over the timed steps; FFAvg pairs add two shared "
                    "atomics (count, distance offset)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 distances, u32/u64 integer bins, f64 transform", "data": "synthetic (seeded generator)",
        "config": batch_config(wl),
        "transform": {"precision": args.precision, "tolerance": args.tolerance,
                      "fp64_fraction": fp64_cols / float(n * nq), "max_rel_diff_vs_fp64_transform": tc_diff,
                      "note": "exact-accumulation tensor-core transform (int8 digits, s32 sums) over shared "
                              "Taylor tables; FP64 for the (structure, q) values whose rigorous bound exceeds "
                              "the tolerance"},
        "plain_sequential": {"value": plain_value, "unit": UNIT, "speedup_batched_vs_plain": value / plain_value,
                             "max_rel_diff_vs_batched": plain_diff,
                             "note": f"{n} resident structures, one ausaxs_gpu_structure_profile call each, in sequence"},
        "autotune": {"choice": choice, "candidate": _capi.Batch.candidate(choice),
                     "pair_ms_per_candidate": [round(float(x), 3) for x in cand_ms[:7]]},
        "l2": "256 MiB buffer written between timed steps (outside the events)",
        "parallelism": f"replicas x{world}",
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                "max_rel_diff_vs_fresh_batch": e2e_diff,
                "note": ("C ABI from pinned host records, host clock: per step ausaxs_gpu_batch_set_points (all "
                         f"{n} structures' coordinates and excluded-volume charges; two poses alternating) + "
                         "ausaxs_gpu_batch_profile (q up, graph replay, every I(q) down, synchronised)"),
                "new_batch_per_step": {"value": e2e_new, "unit": UNIT,
                                       "p50_ms": 1e3 * float(np.percentile(lat_new, 50)),
                                       "note": "ausaxs_gpu_batch_create + _profile + _destroy per step (census, "
                                               "plans and graph capture inside)"}},
        "gpu_launches": int(launches),
        "roofline": roof,
        "clocks": clocks,
        "peaks_source": peak_kind,
    }
    B.close()
    ctx.close()
    del flush
    if args.workload == "cfg3" and not args.no_serving:
        line["serving"] = serving_measure(args, rank, world, local_rank, compact=True)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, det = time_reference_batch(wl, steps=1, warmup=0, n_chunks=16)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, **det} if v is not None else det
    return line


def run_serving(args, rank, world, local_rank):
    return serving_measure(args, rank, world, local_rank, compact=False)


def serving_measure(args, rank, world, local_rank, compact=False):
    """Rigid-body serving: 64 device-resident 8-body assemblies, one random rigid move per request,
    Poisson arrivals at several rates and a closed-loop saturation run; latency from the scheduled
    arrival to the observed completion (host clock).  Also the latency of a move submitted alone (no
    other request in flight), for the largest body of every assembly and for random bodies.
    compact: the figures as a sub-object of another workload's line."""
    import collections

    import torch

    from ausaxs_b200 import _capi, hist, synth

    torch.cuda.set_device(local_rank)
    chains = args.chains
    nq = 400
    q = np.linspace(0.005, 0.5, nq)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, args.serve_precision, 1e-4 if args.serve_precision != 1 else 1e-5)
    rng = np.random.default_rng(4 + rank)
    t_gen = time.perf_counter()
    asm = [synth.assembly(1000 * rank + 40 + c) for c in range(chains)]
    t_gen = time.perf_counter() - t_gen
    S = _capi.Server(local_rank, hbm_budget=int(args.hbm_budget_gb * (1 << 30)), max_inflight=4 * chains,
                     slots_per_assembly=2)
    S.set_policy(args.serve_policy)
    ids, sizes, footprints = [], [], []
    t_admit = time.perf_counter()
    for A in asm:
        atoms = [hist.pack(b, f, True) for b, f in zip(A.bodies, A.ff)]
        wats = [np.zeros((0, 4), np.float32) for _ in A.bodies]
        n = sum(len(a) for a in atoms)
        # average excluded-volume charge for a protein-like specific volume of 18 A^3 per atom
        cfg = _capi.HistConfig(_capi.MANAGER_FFAVG, 1, 0.25, 8000, 18.0 * 0.334)
        probe = S.admit(cfg, atoms, wats, q, p, margin=20.0)[0]
        I0, _ = S.wait(S.submit(probe), probe)
        S.release(probe)
        target = I0 * (1 + 0.01 * rng.standard_normal(nq))  # 1 % Gaussian noise on the FP64 profile
        sid, fp = S.admit(cfg, atoms, wats, q, p, target=target, target_err=0.01 * np.abs(I0), margin=20.0)
        ids.append(sid)
        sizes.append([len(a) for a in atoms])
        footprints.append(fp)
    t_admit = time.perf_counter() - t_admit

    def move(sid, body):
        R = synth.random_rotation(rng, 5.0)
        t = rng.standard_normal(3)
        t *= 2.0 * rng.uniform() / max(np.linalg.norm(t), 1e-12)
        c = S.body_center(sid, body)
        return R, c - R @ c + t

    def run(n_req, rate=None):
        """Open loop at `rate` requests/s (Poisson), or closed loop (every free slot refilled) when None."""
        arrivals = collections.deque()
        t = 0.0
        for _ in range(n_req):
            if rate:
                t += rng.exponential(1.0 / rate)
            k = int(rng.integers(0, chains))
            arrivals.append((t, k, int(rng.integers(0, 8))))
        inflight = {}
        lat, done, first, last = [], 0, None, None
        t0 = time.perf_counter()
        while done < n_req:
            now = time.perf_counter() - t0
            while arrivals and (rate is None or arrivals[0][0] <= now):
                ta, k, body = arrivals[0]
                R, tv = move(ids[k], body)
                tk = S.try_submit(ids[k], body, R, tv)
                if tk is None:
                    break
                arrivals.popleft()
                inflight[tk] = (ids[k], ta if rate else now)
                if first is None:
                    first = now
            for tk in S.completed():
                sid, ta = inflight.pop(tk)
                S.poll(tk, sid)
                now = time.perf_counter() - t0
                lat.append(now - ta)
                done += 1
                last = now
        lat = np.array(lat) * 1e3
        return {"rate_offered": rate, "requests": n_req, "moves_per_s": n_req / (last - first),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "mean_ms": float(lat.mean())}

    n_req = args.serve_requests or 5 * chains
    run(4 * chains, None)  # warm-up
    launches0 = S.launches()
    with ClockSampler(local_rank) as clk:
        sat = run(n_req, None)
    sat_launches = S.launches() - launches0
    # whole job: every rank serves its own chains; the job lasts as long as its slowest rank
    sat_total = world * sat["requests"] / max_over_ranks(sat["requests"] / sat["moves_per_s"], world)
    sweep = []
    for frac in (0.25, 0.5, 0.75):
        sweep.append(run(n_req, frac * sat["moves_per_s"]))

    def lone(k, body):
        R, tv = move(ids[k], body)
        t0 = time.perf_counter()
        S.wait(S.submit(ids[k], body, R, tv), ids[k])
        return 1e3 * (time.perf_counter() - t0)

    lone_largest = [lone(k, int(np.argmax(sizes[k]))) for k in range(chains)]
    lone_random = [lone(k, int(rng.integers(0, 8))) for k in range(chains)]
    # pair evaluations of an average move: the moved body against every other body plus its own pairs
    per_move = []
    for sz in sizes:
        tot = sum(sz)
        per_move.append(np.mean([n * (tot - n) + n * (n - 1) / 2 for n in sz]))
    pairs_per_move = float(np.mean(per_move))
    lone_stats = {"largest_body_p50_ms": float(np.percentile(lone_largest, 50)),
                  "largest_body_max_ms": float(np.max(lone_largest)),
                  "random_body_p50_ms": float(np.percentile(lone_random, 50)),
                  "note": "one move submitted with nothing else in flight, submit to result on the host"}
    if compact:
        S.close()
        return {"workload": f"cfg4: {chains} chains x 8-body assemblies, bodies 3k-20k atoms, 400 q, moves <= 5 deg + <= 2 A",
                "moves_per_s_saturated": sat_total, "saturation": sat, "poisson_sweep": sweep, "lone": lone_stats,
                "pairs_per_move_mean": pairs_per_move, "gpu_launches_saturated": int(sat_launches),
                "clocks": clk.summary()}
    line = {
        "metric": "rigid-body moves/s (I(q) + chi2 per move) with p50/p99 latency", "value": sat_total,
        "unit": "moves/s", "n_gpus": world, "steps": args.steps, "warmup": 4, "ms_per_step": 1e3 / sat["moves_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 distances, u64 integer partial histograms, f64 transform and fit",
        "data": "synthetic (seeded generator)",
        "config": {"workload": f"cfg4: {chains} chains x 8-body assemblies, bodies 3k-20k atoms, 400 q, "
                               f"moves <= 5 deg about the body centroid + <= 2 A",
                   "atoms_total": int(sum(sum(s) for s in sizes)), "pairs_per_move_mean": pairs_per_move,
                   "footprint_bytes_total": int(sum(footprints)), "admit_s": t_admit, "generate_s": t_gen,
                   "saturation": sat, "poisson_sweep": sweep, "lone": lone_stats},
        "e2e": {"value": sat_total, "unit": "moves/s", "h2d_bytes_per_step": 96,
                "d2h_bytes_per_step": (nq + 5) * 8, "p50_ms": sat["p50_ms"], "p99_ms": sat["p99_ms"],
                "note": "every request crosses the host ABI: pose in, I(q) and fit out"},
        "gpu_launches": int(sat_launches),
        "clocks": clk.summary(),
    }
    peaks, _ = load_peaks()
    sm_mhz = line["clocks"].get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    atomic_rate, _ = _capi.smem_atomic_rate(local_rank, True)
    # pair evaluations of the saturated run per second of it (every other stage of a request included)
    line["roofline"] = pair_roofline(pairs_per_move, 1e3 / sat["moves_per_s"], sm_mhz, sms, atomic_rate, 2,
                                     INSTR_PER_PAIR)
    line["roofline"]["traffic"] = None
    line["roofline"]["note"] = "pair evaluations of the saturated serving run (moved body x the rest + its own pairs)"
    S.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref_args = argparse.Namespace(steps=1, warmup=0)
        r = run_reference_serving(ref_args, 1)
        line["cpu_baseline"] = r.get("cpu_baseline", {"unavailable": r.get("unavailable")})
    return line


def run_ours(args, rank, world, local_rank):
    import torch

    from ausaxs_b200 import _capi
    from ausaxs_b200.hist import (HistogramManagerMTFFAvg, HistogramManagerMTFFGrid, RHO_WATER)

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream(local_rank)
    ctx = _capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    wl = workload(args.workload, args.subunit, args.atoms)
    m = wl.molecules[0]
    grid = wl.manager == "ffgrid"
    mgr = (HistogramManagerMTFFGrid(m, wl.bin_width, wl.bin_count, ctx) if grid
           else HistogramManagerMTFFAvg(m, True, wl.bin_width, wl.bin_count, ctx))
    cfg = mgr.config()
    A, W, X = mgr._inputs()
    pairs = pair_count(m, grid)
    # precision 2 (default): the exact-accumulation tensor-core transform where it pays off (FP64 for
    # every q whose rigorous error bound exceeds the tolerance, the path's I(q) bar of 1e-4 relative to
    # the FP64 transform), the FP64 transform for small ones
    params = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, args.precision, args.tolerance)
    nq = len(wl.q)
    q_dev = torch.tensor(wl.q, dtype=torch.float64, device=f"cuda:{local_rank}")
    I_dev = torch.zeros(nq, dtype=torch.float64, device=f"cuda:{local_rank}")
    st = _capi.Structure(ctx, A, W, X if grid else None, ff_typed=True)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local_rank}")

    def step():
        st.profile_device(cfg, q_dev, nq, params, I_dev)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
            flush.fill_(1.0)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ctx.enable_timing(True)
        launches0 = ctx.launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                step()
                ends[k].record(stream)
                flush.fill_(float(k))  # L2 flush between steps, outside the timed events
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        k_ms, k_n = ctx.kernel_time(0)
        lat_ms, lat_n = ctx.kernel_time(6)
        ctx.enable_timing(False)
    total_ms = sum(step_ms)
    total_ms = max_over_ranks(total_ms, world)
    value = world * args.steps / (total_ms / 1e3)
    I_gpu = I_dev.cpu().numpy()
    # the same structure through the FP64 transform: deviation of the timed result
    I_64 = torch.zeros_like(I_dev)
    st.profile_device(cfg, q_dev, nq, _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5), I_64)
    torch.cuda.synchronize()
    iq_dev_fp64 = float(np.max(np.abs(I_gpu / I_64.cpu().numpy() - 1)))
    # the q values the timed transform evaluated in FP64 (the tensor-core path re-evaluates every q whose
    # error bound exceeds the tolerance; the automatic choice takes FP64 for small transforms)
    h_chk = mgr.calculate_all()
    h_chk.precision, h_chk.tolerance = args.precision, args.tolerance
    h_chk.debye_transform(wl.q)
    fp64_q = ctx.fp64_columns()

    # end to end through the host C ABI with pinned buffers
    pin_a = torch.from_numpy(A).pin_memory()
    pin_w = torch.from_numpy(W).pin_memory()
    pin_x = torch.from_numpy(X).pin_memory() if grid else None
    pin_q = torch.from_numpy(np.ascontiguousarray(wl.q)).pin_memory()
    pin_I = torch.zeros(nq, dtype=torch.float64).pin_memory()
    import ctypes as C

    L = _capi.load()

    def e2e_step():
        _capi.check(L.ausaxs_gpu_profile(ctx.h, C.byref(cfg), _capi.devptr(pin_a, C.c_float), len(A),
                                         _capi.devptr(pin_w, C.c_float), len(W),
                                         _capi.devptr(pin_x, C.c_float) if grid else C.cast(0, C.POINTER(C.c_float)),
                                         len(X) if grid else 0, _capi.devptr(pin_q), nq, C.byref(params),
                                         _capi.devptr(pin_I), C.cast(0, C.POINTER(C.c_double))))

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    if world > 1:
        torch.distributed.barrier()
    lat = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        lat.append(time.perf_counter() - t0)
    e2e_total = sum(lat)
    e2e_total = max_over_ranks(e2e_total, world)
    e2e = world * args.steps / e2e_total
    e2e_match = float(np.max(np.abs(pin_I.numpy() / I_gpu - 1)))

    peaks, peak_kind = load_peaks()
    kernel_ms = k_ms / args.steps  # all pair-kernel launches of one profile
    # the grid dummies' self pairs go to the lattice kernel when it launched (class 6)
    nx = len(m.exv) if (grid and m.exv is not None) else 0
    lattice_pairs = nx * (nx - 1) // 2 if lat_n else 0
    pair_rate = (pairs - lattice_pairs) / (kernel_ms / 1e3)
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    atomic_rate, _ = _capi.smem_atomic_rate(local_rank, True)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 distances, u32/u64 integer bins, f64 transform", "data": "synthetic (seeded generator)",
        "config": {"workload": wl.name, "atoms": m.size_atom(), "waters": m.size_water(),
                   "exv": 0 if m.exv is None or not grid else len(m.exv), "pairs_per_profile": pairs,
                   "bin_width": wl.bin_width, "q_points": nq, "manager": wl.manager,
                   "transform": {"precision": args.precision, "tolerance": args.tolerance,
                                 "max_rel_diff_vs_fp64_transform": iq_dev_fp64,
                                 "fp64_q_fraction": fp64_q / nq},
                   "l2": "256 MiB buffer written between timed steps (outside the events)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(A.nbytes + W.nbytes + (X.nbytes if grid else 0) + pin_q.numel() * 8),
                "d2h_bytes_per_step": int(nq * 8 + 8), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)), "max_rel_diff_vs_resident": e2e_match},
        "gpu_launches": int(launches),
        "roofline": dict(pair_roofline(pairs - lattice_pairs, kernel_ms, sm_mhz, sms, atomic_rate, 2, INSTR_PER_PAIR),
                         traffic=None, kernel_launches_per_step=k_n / args.steps,
                         note="pair evaluations of the pair kernel per second of its launches (the grid dummies' "
                              "self pairs, when the lattice kernel takes them, are not counted)"),
        "lattice": ({"kernel": "lattice_kernel", "ms_per_step": lat_ms / args.steps, "dummy_pairs": lattice_pairs,
                     "pair_equivalent_per_s": lattice_pairs / (lat_ms / args.steps / 1e3) if lat_ms else None,
                     "note": "the dummies' self pairs by the occupancy autocorrelation (integer popcounts); the "
                             "accumulators equal the pair kernel's"} if lat_n else None),
        "clocks": clocks,
        "peaks_source": peak_kind,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, det = time_reference(m, wl, steps=1, warmup=0)
        if v is not None:
            line["cpu_baseline"] = {"value": v, "unit": UNIT, **det}
        else:
            line["cpu_baseline"] = det
    st.close()
    ctx.close()
    return line


def run_reference_serving(args, world):
    """The reference's answer to a rigid move of an FFAvg assembly: a full calculate_all() of the
    moved assembly plus its transform (its partial manager exists for the Simple model only), timed on
    one assembly of the serving workload."""
    from ausaxs_b200 import synth
    from oracle import py as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    threads = max(1, (os.cpu_count() or 2) - 1)
    O.ref(threads)
    O.ref_set_axes(0.25, 8000, 1e-4, 1.0)
    O.ref_set_simple_exv(False)
    A = synth.assembly(40)
    xyz = np.concatenate(A.bodies)
    ff = np.concatenate(A.ff)
    w = np.concatenate(A.weights)
    rm = O.RefMolecule(xyz, w, ff, np.zeros((0, 3)), np.zeros(0), volume=18.0 * len(xyz))
    rm.set_manager("ffavg")
    times = []
    for it in range(args.warmup + args.steps):
        h = rm.calculate()
        _, _, _, t_debye = h.debye()
        if it >= args.warmup:
            times.append(h.seconds + t_debye * (400 / 200.0))
    v = 1.0 / statistics.median(times)
    det = {"cores": threads, "kind": "reference",
           "sample": f"one {len(xyz)}-atom 8-body assembly: full FFAvg calculate_all() + debye_transform() per move"}
    return {"impl": "reference", "metric": "rigid-body moves/s (I(q) + chi2 per move) with p50/p99 latency",
            "value": v, "unit": "moves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 distances, f64 bins and transform (reference CPU)", "data": "synthetic (seeded generator)",
            "config": {"workload": "cfg4 (one assembly)", "manager": "ffavg"},
            "cpu_baseline": {"value": v, "unit": "moves/s", **det},
            "e2e": {"value": v, "unit": "moves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


GRID_METRIC = "excluded-volume grids/s (RawGridExv dummies + grid volume of one structure)"
GRID_UNIT = "grids/s"


def grid_workload():
    """The 50k-atom + 10k-water structure of the WAXS configuration; its 1 A molecular grid."""
    from ausaxs_b200 import synth

    m = synth.cfg1().molecules[0]
    return m, "gridexv: molecular grid of the 50k-atom + 10k-water structure (1 A cells, rvol 2.15 A)"


def grid_shape(m):
    """Cells of the expanded grid (the same axes rule as the device code) for the traffic model."""
    lo = np.minimum(0.0, np.minimum(m.atoms.min(0), m.waters.min(0)))
    hi = np.maximum(0.0, np.maximum(m.atoms.max(0), m.waters.max(0)))
    diff = hi - lo
    scaling = 1.0 if np.any(diff < 50) else 0.25
    e = np.maximum(0.5 * diff * scaling, 2.14 + 1.71 - 0.35 + 3.0)
    bins = np.ceil(hi + e + 1.0) - np.floor(lo - e - 1.0)
    return int(np.prod(bins))


def run_gridexv(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from ausaxs_b200 import _capi

    torch.cuda.set_device(local_rank)
    dev = torch.device(f"cuda:{local_rank}")
    stream = torch.cuda.Stream(local_rank)
    ctx = _capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    m, name = grid_workload()
    A, W, _ = m.compact_ff()
    cells = grid_shape(m)
    a_d, w_d = torch.from_numpy(A).to(dev), torch.from_numpy(W).to(dev)
    n0 = len(_capi.grid_exv(ctx, A, W)[0])
    out = torch.zeros((n0, 4), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def step():
        return _capi.grid_exv_device(ctx, a_d, len(A), w_d, len(W), out, n0)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ctx.enable_timing(True)
        launches0 = ctx.launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                n, vol = step()
                ends[k].record(stream)
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        k_ms, k_n = ctx.kernel_time(4)
        ctx.enable_timing(False)
    total_ms = max_over_ranks(sum(s.elapsed_time(e) for s, e in zip(starts, ends)), world)
    value = world * args.steps / (total_ms / 1e3)

    # end to end through the host C ABI: pinned records in, pinned dummies out
    pin_a = torch.from_numpy(A).pin_memory()
    pin_w = torch.from_numpy(W).pin_memory()
    pin_o = torch.zeros((n0, 4), dtype=torch.float32).pin_memory()
    L = _capi.load()
    nn, vv = C.c_int64(0), C.c_double(0)

    def e2e_step():
        _capi.check(L.ausaxs_gpu_grid_exv(ctx.h, _capi.devptr(pin_a, C.c_float), len(A), _capi.devptr(pin_w, C.c_float),
                                          len(W), 1, _capi.devptr(pin_o, C.c_float), n0, C.byref(nn), C.byref(vv)))

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    lat = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        lat.append(time.perf_counter() - t0)
    e2e = world * args.steps / max_over_ranks(sum(lat), world)
    same = bool(np.array_equal(pin_o.numpy(), out.cpu().numpy())) and nn.value == n and vv.value == vol

    peaks, peak_kind = load_peaks()
    kernel_ms = k_ms / args.steps
    # algorithmic bytes of one grid: clear the cell words, two sweeps over them (count, write), the
    # points read by the three point kernels, the dummies written
    alg = cells * 4 * 3 + (len(A) + len(W)) * 16 + len(A) * 16 * 2 + n * 16
    achieved = alg / (kernel_ms / 1e3) / 1e9
    line = {
        "metric": GRID_METRIC, "value": value, "unit": GRID_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 cell distances, u32 cell flags", "data": "synthetic (seeded generator)",
        "config": {"workload": name, "atoms": m.size_atom(), "waters": m.size_water(), "cells": cells,
                   "dummies": int(n), "volume_A3": vol, "l2": f"grid of {cells * 4 / 1e6:.0f} MB stays in L2 (no flush: "
                   "the step is bound by launch and synchronisation latency, not DRAM)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": GRID_UNIT, "h2d_bytes_per_step": int(A.nbytes + W.nbytes),
                "d2h_bytes_per_step": int(n * 16 + 16), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)), "same_as_resident": same},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "grid excluded-volume kernels (class 4)", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes": int(alg), "kernel_ms_per_step": kernel_ms,
                     "kernel_intervals_per_step": k_n / args.steps,
                     "note": "two event intervals per step (before and after the count read-back)"},
        "clocks": clk.summary(),
        "peaks_source": peak_kind,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_grid(m)
    ctx.close()
    return line


def reference_grid(m, steps: int = 1, warmup: int = 0):
    from oracle import py as O

    if not O.ref_available():
        return {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    O.ref(1)
    ts = []
    for it in range(warmup + steps):
        t, n, vol = O.ref_grid_exv_seconds(m.atoms, m.ff_types, m.waters)
        if it >= warmup:
            ts.append(t)
    v = 1.0 / statistics.median(ts)
    return {"value": v, "unit": GRID_UNIT, "cores": 1, "kind": "reference", "dummies": n, "volume_A3": vol,
            "sample": "the whole structure: Molecule construction, grid creation and expansion, RawGridExv sweep "
                      "(single-threaded in the reference)"}


HYD_METRIC = "hydration shells/s (Molecule::generate_new_hydration, RadialHydration, fresh grid, one structure)"
HYD_UNIT = "shells/s"


def hydrate_workload():
    """The 50k-atom globule of the WAXS configuration, hydrated from scratch (its atoms only)."""
    from ausaxs_b200 import synth

    m = synth.cfg1().molecules[0]
    xyz = np.ascontiguousarray(np.asarray(m.atoms, np.float64))
    ff = np.ascontiguousarray(np.asarray(m.ff_types, np.int32))
    return xyz, ff, "hydrate: RadialHydration of the 50k-atom globule (1 A grid, 26 directions, no noise)"


def run_hydrate(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from ausaxs_b200 import _capi

    torch.cuda.set_device(local_rank)
    dev = torch.device(f"cuda:{local_rank}")
    stream = torch.cuda.Stream(local_rank)
    ctx = _capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    xyz, ff, name = hydrate_workload()
    axes = _capi.hydrate_axes(xyz)
    cells = int(np.prod(axes[3:]))
    w0, c0, _ = _capi.hydrate(ctx, xyz, ff)
    cap = len(w0) + 1024
    a_d, f_d = torch.from_numpy(xyz).to(dev), torch.from_numpy(ff).to(dev)
    out = torch.zeros((cap, 3), dtype=torch.float64, device=dev)
    cand = torch.zeros(cap, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()

    def step():
        return _capi.hydrate_device(ctx, a_d, f_d, len(xyz), axes, out, cap, cand)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ctx.enable_timing(True)
        launches0 = ctx.launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                n, rounds = step()
                ends[k].record(stream)
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        k_ms, k_n = ctx.kernel_time(5)
        ctx.enable_timing(False)
    total_ms = max_over_ranks(sum(s_.elapsed_time(e) for s_, e in zip(starts, ends)), world)
    value = world * args.steps / (total_ms / 1e3)
    same = n == len(w0) and bool(np.array_equal(out[:n].cpu().numpy(), w0))

    # end to end through the host C ABI: pinned atoms and types in, pinned waters out
    pin_a = torch.from_numpy(xyz).pin_memory()
    pin_f = torch.from_numpy(ff).pin_memory()
    pin_o = torch.zeros((cap, 3), dtype=torch.float64).pin_memory()
    pin_c = torch.zeros(cap, dtype=torch.int64).pin_memory()
    L = _capi.load()
    nn, rr = C.c_int64(0), C.c_int32(0)

    def e2e_step():
        _capi.check(L.ausaxs_gpu_hydrate(ctx.h, _capi.devptr(pin_a, C.c_double), _capi.devptr(pin_f, C.c_int32),
                                         len(xyz), None, None, 0, _capi.devptr(pin_o, C.c_double), cap, C.byref(nn),
                                         _capi.devptr(pin_c, C.c_int64), C.byref(rr)))

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    lat = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        lat.append(time.perf_counter() - t0)
    e2e = world * args.steps / max_over_ranks(sum(lat), world)
    same = same and nn.value == n and bool(np.array_equal(pin_o.numpy()[:n], w0))

    peaks, peak_kind = load_peaks()
    kernel_ms = k_ms / args.steps
    surv, _ = _capi.hydration_stats(ctx)
    # algorithmic bytes of one shell, as a one-round resolution would touch them: atoms and types read,
    # the cell grid written once, one cell read and one atom read per candidate, the 79 probe cells
    # (state byte and two key words) of every candidate that survives the static tests, the waters
    # and their indices written
    alg = len(xyz) * 28 + cells + 26 * len(xyz) * 25 + surv * 79 * 17 + n * 32
    achieved = alg / (kernel_ms / 1e3) / 1e9
    line = {
        "metric": HYD_METRIC, "value": value, "unit": HYD_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 positions and distances, u8 cell states, u64 candidate keys",
        "data": "synthetic (seeded generator)",
        "config": {"workload": name, "atoms": len(xyz), "cells": cells, "waters": int(n), "rounds": int(rounds),
                   "candidates_surviving_static_tests": surv,
                   "l2": f"grid of {cells / 1e6:.1f} MB and keys of {cells * 16 / 1e6:.0f} MB stay in L2 (no flush: the "
                         "step is bound by the rounds' launch and read-back latency, not DRAM)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": HYD_UNIT, "h2d_bytes_per_step": int(xyz.nbytes + ff.nbytes),
                "d2h_bytes_per_step": int(n * 32 + 16), "p50_ms": 1e3 * float(np.percentile(lat, 50)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)), "same_as_resident": same},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": "hydration kernels (class 5)", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes": int(alg), "kernel_ms_per_step": kernel_ms,
                     "kernel_intervals_per_step": k_n / args.steps,
                     "note": "latency-bound: the rounds (one kernel each) run in batches of 16 between "
                             "read-backs; the intervals exclude the host gaps at the read-backs"},
        "clocks": clk.summary(),
        "peaks_source": peak_kind,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_hydrate(xyz, ff)
    ctx.close()
    return line


def reference_hydrate(xyz, ff, steps: int = 1, warmup: int = 0):
    from oracle import py as O

    if not O.ref_available():
        return {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    O.ref(1)
    ts = []
    n = 0
    for it in range(warmup + steps):
        m = O.RefMolecule(xyz, np.ones(len(xyz)), ff, np.zeros((0, 3)), np.zeros(0))
        _, w, _, _, t = m.hydrate(None, True, 1)
        n = len(w)
        if it >= warmup:
            ts.append(t)
    v = 1.0 / statistics.median(ts)
    return {"value": v, "unit": HYD_UNIT, "cores": 1, "kind": "reference", "waters": n,
            "sample": "the whole structure: grid creation and expansion, RadialHydration over every atom "
                      "(single-threaded in the reference)"}


FIT_METRIC = "fits/s (coordinates -> histogram -> SmartFitter fit of cw by golden-section search)"
FIT_UNIT = "fits/s"
# the reference's q axis (constants::axes::q_axis: 200 bins on [1e-4, 1]) below qmax = 0.5: 99 points
FIT_Q = 1e-4 + 0.0049995 * np.arange(99)


def fit_data(I, seed=17):
    """Synthetic measurement from a model curve: scaled, offset, 1 % Gaussian noise."""
    r = np.random.default_rng(seed)
    y0 = 2.5 * I + 0.002 * np.abs(I).max()
    sigma = 0.01 * np.abs(y0) + 1e-6 * np.abs(y0).max()
    return y0 + sigma * r.standard_normal(len(I)), sigma


def run_fit(args, rank, world, local_rank):
    import ctypes as C

    import torch

    from ausaxs_b200 import _capi
    from ausaxs_b200._capi import HistResult
    from ausaxs_b200.hist import NFF, HistogramManagerMTFFAvg

    torch.cuda.set_device(local_rank)
    dev = torch.device(f"cuda:{local_rank}")
    stream = torch.cuda.Stream(local_rank)
    ctx = _capi.Context(local_rank)
    ctx.set_stream(stream.cuda_stream)
    wl = workload("cfg0")
    m = wl.molecules[0]
    mgr = HistogramManagerMTFFAvg(m, True, wl.bin_width, wl.bin_count, ctx)
    cfg = mgr.config()
    A, W, _ = mgr._inputs()
    h = mgr.calculate_all()
    h.apply_water_scaling_factor(1.3)
    q = np.ascontiguousarray(FIT_Q)
    _, I_true = h.debye_transform(q)
    y, sigma = fit_data(I_true)
    base = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 0.0)
    opt = _capi.FitOptions(0, 0.0, 0.0, 1e-4)
    st = _capi.Structure(ctx, A, W, None, ff_typed=True)
    q_d, y_d, s_d = (torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (q, y, sigma))
    torch.cuda.synchronize()

    def step():
        return st.fit_device(cfg, q_d, y_d, s_d, len(q), base, opt)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ctx.enable_timing(True)
        launches0 = ctx.launches
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        with ClockSampler(local_rank) as clk:
            torch.cuda.synchronize()
            for k in range(args.steps):
                starts[k].record(stream)
                r = step()
                ends[k].record(stream)
            torch.cuda.synchronize()
        launches = ctx.launches - launches0
        k_ms, k_n = ctx.kernel_time(0)
        ctx.enable_timing(False)
    total_ms = max_over_ranks(sum(s_.elapsed_time(e) for s_, e in zip(starts, ends)), world)
    value = world * args.steps / (total_ms / 1e3)

    # end to end through the host C ABI: coordinates -> ausaxs_gpu_histogram -> ausaxs_gpu_fit
    L = _capi.load()
    nb = wl.bin_count
    bufs = {k: np.zeros(n) for k, n in [("aa", NFF * NFF * nb), ("aw", NFF * nb), ("ww", nb), ("tot", nb), ("d_axis", nb),
                                         ("d_axis_ax", nb), ("d_axis_xx", nb)]}
    res = HistResult()
    for k, v in bufs.items():
        setattr(res, k, _capi.dptr(v))
    out = _capi.FitResult()

    def e2e_step():
        _capi.check(L.ausaxs_gpu_histogram(ctx.h, C.byref(cfg), _capi.fptr(A), len(A), _capi.fptr(W), len(W),
                                           _capi.fptr(None), 0, C.byref(res)))
        _capi.check(L.ausaxs_gpu_fit(ctx.h, C.byref(cfg), C.byref(res), _capi.dptr(q), _capi.dptr(y), _capi.dptr(sigma),
                                     len(q), C.byref(base), C.byref(opt), C.byref(out), _capi.dptr(None)))

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    lat = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        lat.append(time.perf_counter() - t0)
    e2e = world * args.steps / max_over_ranks(sum(lat), world)
    pairs = pair_count(m, False)
    peaks, peak_kind = load_peaks()
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    issue_peak = sms * 4 * sm_mhz * 1e6 * 32 / INSTR_PER_PAIR
    pair_rate = pairs / (k_ms / args.steps / 1e3)
    line = {
        "metric": FIT_METRIC, "value": value, "unit": FIT_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 distances, integer bins, f64 transform and fit", "data": "synthetic (seeded generator)",
        "config": {"workload": "fit: cfg0 structure (5k atoms + 1k waters, FFAvg, 0.25 A bins), 99 q on the "
                               "reference's axis, cw fitted in [0, 10] to 1e-4",
                   "fitted": {"cw": r.value, "a": r.a, "b": r.b, "chi2": r.chi2, "evaluations": r.evaluations},
                   "same_e2e": bool(out.value == r.value and out.evaluations == r.evaluations),
                   "l2": "inputs of 0.1 MB stay in L2 (the step is bound by launch latency)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e, "unit": FIT_UNIT, "h2d_bytes_per_step": int(A.nbytes + W.nbytes + 3 * q.nbytes),
                "d2h_bytes_per_step": int(8 * (NFF * NFF + NFF + 3) * h.max_bin + 56),
                "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99))},
        "gpu_launches": int(launches),
        "roofline": {"bound": "issue", "kernel": "pairhist_kernel", "achieved": pair_rate / 1e9, "peak": issue_peak / 1e9,
                     "unit": "Gpair/s", "frac": pair_rate / issue_peak, "traffic": None,
                     "note": "a 5k-atom histogram is launch-latency bound; the fit kernel itself is one CTA"},
        "clocks": clocks,
        "peaks_source": peak_kind,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_fit(steps=1, warmup=0)
    st.close()
    ctx.close()
    return line


def reference_fit(steps: int, warmup: int):
    """The reference: calculate_all() of the cfg0 structure, then SmartFitter::fit() of cw."""
    from oracle import py as O

    if not O.ref_available():
        return {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    threads = max(1, (os.cpu_count() or 2) - 1)
    O.ref(threads)
    wl = workload("cfg0")
    m = wl.molecules[0]
    O.ref_set_axes(wl.bin_width, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(False)
    rm = O.RefMolecule(m.atoms, m.weights, m.ff_types, m.waters, m.water_weights, volume=m.volume)
    rm.set_manager("ffavg")
    ts = []
    for it in range(warmup + steps):
        h = rm.calculate()
        q, I, _, _ = h.debye(1.3, 1.0, 1.0, 0.0, 0.0)
        y, sigma = fit_data(I)
        h.debye(1.0, 1.0, 1.0, 0.0, 0.0)
        h.fit(0, q, y, sigma)
        if it >= warmup:
            ts.append(h.seconds + h.fit_seconds)
    v = 1.0 / statistics.median(ts)
    return {"value": v, "unit": FIT_UNIT, "cores": threads, "kind": "reference",
            "sample": "the whole workload: calculate_all() of the 5k-atom structure (thread pool) and "
                      "SmartFitter::fit() of cw (Golden, single-threaded)"}


SYM_METRIC = "symmetric histograms/s (icosahedral 60-mer through SimpleCalculator jobs, Simple model)"
SYM_UNIT = "histograms/s"


def symmetry_setup(seed: int = 21, subunit: int = 8333):
    """cfg2's shell as one body with 60-fold icosahedral symmetry: the job list SymmetryManagerMT issues
    (SymmetryManagerMT.cpp:37-136) for it, and the expanded structure.  Point sets are float32
    {x, y, z, w} records; jobs are (a, b or None, scaling, merge id) over them."""
    from ausaxs_b200 import synth

    cos_half = 1.0 - 1.0 / 36.0
    sub, ff = synth.globule(seed, subunit, r_in=120.0, r_out=150.0, cone_cos=cos_half)
    R = synth.icosahedral_rotations()
    w = synth.ff_charge(ff)
    copies = [np.column_stack([sub @ r.T, w]).astype(np.float32) for r in R]
    xyz = np.concatenate([c[:, :3] for c in copies]).astype(np.float64)
    wat = synth.waters(seed + 1, xyz, np.tile(ff, len(R)), 60000)
    waters = np.column_stack([wat, np.full(len(wat), synth.ff_charge([synth.FF_WATER])[0])]).astype(np.float32)
    sets = copies + [waters]
    W = len(copies)
    # classes of copy pairs with the same relative rotation up to inversion (PairScheduleUtil.cpp:33-58):
    # representative (0, k) for the first k of each class, scaling = the class size
    key = lambda M: tuple(np.round(M.ravel() * 1e4).astype(np.int64))
    classes = {}
    for i in range(W):
        for j in range(i + 1, W):
            D = R[j].T @ R[i]
            kk = min(key(D), key(D.T))
            if kk not in classes:
                classes[kk] = [i, j, 0]
            classes[kk][2] += 1
    jobs = [(0, None, W, 0), (W, 0, 1, 1)]  # the body once with scaling 1 + copies; waters x body
    jobs += [(i, j, n, 0) for i, j, n in classes.values()]
    jobs += [(W, k, 1, 1) for k in range(1, W)]  # waters x every copy
    jobs += [(W, None, 1, 1)]  # waters
    return sets, jobs, np.concatenate(copies), waters


def symmetry_pairs(sets, jobs):
    n = [len(x) for x in sets]
    return sum(n[a] * (n[a] - 1) // 2 if b is None else n[a] * n[b] for a, b, _, _ in jobs)


def run_symmetry(args, rank, world, local_rank):
    import torch

    from ausaxs_b200 import _capi, hist

    torch.cuda.set_device(local_rank)
    ctx = _capi.Context(local_rank)
    sets, jobs, atoms, waters = symmetry_setup()
    bw = 0.1

    def step():
        calc = _capi.Calculator(ctx, bw, 8000)
        for a, b, sc, m in jobs:
            if b is None:
                calc.enqueue_calculate_self(sets[a], sc, m)
            else:
                calc.enqueue_calculate_cross(sets[a], sets[b], sc, m)
        out = calc.run()
        calc.close()
        return out

    for _ in range(args.warmup):
        out = step()
    launches0 = ctx.launches
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            out = step()
        t = time.perf_counter() - t0
    launches = ctx.launches - launches0
    t = max_over_ranks(t, world)
    value = world * args.steps / t
    # the plain Simple histogram of the expanded structure (HistogramManagerMT), timed the same way
    m = hist.Molecule(atoms=atoms[:, :3].astype(np.float64), weights=atoms[:, 3], waters=waters[:, :3].astype(np.float64),
                      water_weights=waters[:, 3])
    mgr = hist.HistogramManagerMT(m, True, bw, 8000, ctx)
    h = mgr.calculate_all()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        h = mgr.calculate_all()
    t_plain = (time.perf_counter() - t0) / max(1, args.steps // 2)
    aa = out["self"][0][0] + out["cross"][0][0]
    n = min(len(aa), len(h.get_aa_counts()))
    plain_aa = np.zeros(len(aa))
    plain_aa[:len(h.get_aa_counts())] = h.get_aa_counts()
    dev = float(np.abs(aa - plain_aa).sum() / np.abs(plain_aa).sum())
    pairs = symmetry_pairs(sets, jobs)
    line = {
        "metric": SYM_METRIC, "value": value, "unit": SYM_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 distances, integer bins, f64 results", "data": "synthetic (seeded generator)",
        "config": {"workload": "symmetry: cfg2 shell as one 8333-atom body with icosahedral symmetry (60 copies) + "
                               "60k waters, Simple weights, 0.1 A bins",
                   "jobs": len(jobs), "pair_classes": len(jobs) - 62, "pairs_per_step": int(pairs),
                   "pairs_plain": int(len(atoms) * (len(atoms) - 1) // 2 + len(atoms) * len(waters) +
                                      len(waters) * (len(waters) - 1) // 2),
                   "plain_ms": 1e3 * t_plain, "speedup_vs_plain": t_plain / (t / args.steps),
                   "aa_l1_rel_diff_vs_plain": dev,
                   "timing": "wall clock around the host-pointer calls (points uploaded, results read back every step)",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": value, "unit": SYM_UNIT, "h2d_bytes_per_step": int(sum(x.nbytes for x in sets)),
                "d2h_bytes_per_step": int(4 * 3 * 8000 * 8)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_symmetry(sets, jobs, bw)
    ctx.close()
    return line


def reference_symmetry(sets, jobs, bw):
    """The reference's SimpleCalculator on the body's jobs (self and the pair classes, no waters),
    scaled by the pairs of the whole job list."""
    from oracle import py as O

    if not O.ref_available():
        return {"unavailable": "reference build oracle/_ref/libausaxs_ref.so not present"}
    threads = max(1, (os.cpu_count() or 2) - 1)
    O.ref(threads)
    O.ref_set_axes(bw, 8000, 1e-4, 0.5)
    sample = [j for j in jobs if j[0] < len(sets) - 1 and (j[1] is None or j[1] < len(sets) - 1)]
    t0 = time.perf_counter()
    O.ref_calculator(sets, sample)
    t = time.perf_counter() - t0
    frac = symmetry_pairs(sets, sample) / symmetry_pairs(sets, jobs)
    return {"value": frac / t, "unit": SYM_UNIT, "cores": threads, "kind": "reference",
            "sample": f"the body's self and pair-class jobs ({frac:.3f} of the pairs), time scaled by pairs"}


def run_atomics_peak(args, rank, world, local_rank):
    """Shared-memory atomic throughput of the device (the second bound of the pair kernel's roofline)."""
    import torch

    from ausaxs_b200 import _capi

    torch.cuda.set_device(local_rank)
    runs = {True: [], False: []}
    with ClockSampler(local_rank) as clk:
        for _ in range(args.warmup + args.steps):
            for cf in (True, False):
                runs[cf].append(_capi.smem_atomic_rate(local_rank, cf))
    cf = [r for r, _ in runs[True][args.warmup:]]
    rnd = [r for r, _ in runs[False][args.warmup:]]
    clocks = clk.summary()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    v = statistics.median(cf)
    return {"metric": "shared-memory 32-bit atomics/s (conflict-free lanes)", "value": v, "unit": "atomics/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median([m for _, m in runs[True][args.warmup:]]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (generated bins)",
            "config": {"workload": "atomics-peak: every SM full of 512-thread CTAs, 4,096-word shared arrays"},
            "random_bins": statistics.median(rnd),
            "per_sm_per_clock": v / (sms * sm_mhz * 1e6), "random_bins_per_sm_per_clock": statistics.median(rnd) / (sms * sm_mhz * 1e6),
            "clocks": clocks, "gpu_launches": 2 * 2 * (args.warmup + args.steps)}


def run_reference(args, rank, world):
    if args.workload == "atomics-peak":
        return {"impl": "reference", "unavailable": "a device measurement: the reference has no GPU code"}
    if args.workload == "symmetry":
        sets, jobs, _, _ = symmetry_setup()
        det = reference_symmetry(sets, jobs, 0.1)
        if "unavailable" in det:
            return {"impl": "reference", **det}
        v = det["value"]
        return {"impl": "reference", "metric": SYM_METRIC, "value": v, "unit": SYM_UNIT, "n_gpus": world,
                "steps": 1, "warmup": 0, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 distances, f64 bins (reference CPU)",
                "data": "synthetic (seeded generator)", "config": {"workload": "symmetry (icosahedral 60-mer)"},
                "cpu_baseline": det, "e2e": {"value": v, "unit": SYM_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "fit":
        det = reference_fit(steps=args.steps, warmup=args.warmup)
        if "unavailable" in det:
            return {"impl": "reference", **det}
        v = det["value"]
        return {"impl": "reference", "metric": FIT_METRIC, "value": v, "unit": FIT_UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (reference CPU)",
                "data": "synthetic (seeded generator)", "config": {"workload": "fit (cfg0 structure, cw)"},
                "cpu_baseline": det, "e2e": {"value": v, "unit": FIT_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "cfg4":
        return run_reference_serving(args, world)
    if args.workload == "hydrate":
        xyz, ff, name = hydrate_workload()
        det = reference_hydrate(xyz, ff, steps=args.steps, warmup=args.warmup)
        if "unavailable" in det:
            return {"impl": "reference", **det}
        v = det["value"]
        return {"impl": "reference", "metric": HYD_METRIC, "value": v, "unit": HYD_UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (reference CPU)",
                "data": "synthetic (seeded generator)", "config": {"workload": name}, "cpu_baseline": det,
                "e2e": {"value": v, "unit": HYD_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "gridexv":
        m, name = grid_workload()
        det = reference_grid(m, steps=args.steps, warmup=args.warmup)
        if "unavailable" in det:
            return {"impl": "reference", **det}
        v = det["value"]
        return {"impl": "reference", "metric": GRID_METRIC, "value": v, "unit": GRID_UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (reference CPU)",
                "data": "synthetic (seeded generator)", "config": {"workload": name}, "cpu_baseline": det,
                "e2e": {"value": v, "unit": GRID_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    wl = workload(args.workload)
    if args.workload == "cfg3":
        v, det = time_reference_batch(wl, steps=args.steps, warmup=args.warmup)
        if v is None:
            return {"impl": "reference", **det}
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * det["seconds"] / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 distances, f64 bins and transform (reference CPU)",
                "data": "synthetic (seeded generator)", "config": batch_config(wl),
                "cpu_baseline": {"value": v, "unit": UNIT, **det},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if not args.no_serving:
            r = run_reference_serving(argparse.Namespace(steps=2, warmup=0), world)
            line["serving"] = {k: r.get(k) for k in ("value", "unit", "cpu_baseline", "unavailable") if k in r}
        return line
    v, det = time_reference(wl.molecules[0], wl, steps=args.steps, warmup=args.warmup, target_pairs=2e9)
    if v is None:
        return {"impl": "reference", **det}
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 distances, f64 bins and transform (reference CPU)",
            "data": "synthetic (seeded generator)", "config": {"workload": wl.name, "manager": wl.manager},
            "cpu_baseline": {"value": v, "unit": UNIT, **det},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4", "gridexv", "fit", "symmetry",
                                                              "hydrate", "atomics-peak"])
    ap.add_argument("--chains", type=int, default=64)
    ap.add_argument("--hbm-budget-gb", type=float, default=40.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="cfg3: skip the serving sub-object")
    ap.add_argument("--serve-requests", type=int, default=0, help="serving: requests per load point (default 5 x chains)")
    ap.add_argument("--serve-policy", type=int, default=2,
                    help="serving: k > 0 submission order over k streams (default 2), 0 concurrent per-assembly "
                         "streams (small moves first)")
    ap.add_argument("--serve-precision", type=int, default=1, choices=[1, 2, 3],
                    help="serving: the per-move transform (1 FP64, 3 exact-accumulation tensor cores, 2 automatic)")
    ap.add_argument("--subunit", type=int, default=0, help="cfg2: atoms per subunit (default 8333; smaller for profiling)")
    ap.add_argument("--atoms", type=int, default=0, help="cfg1: atoms of the globule (default 50000; smaller for profiling)")
    ap.add_argument("--structures", type=int, default=0,
                    help="cfg3: the first structures of the seeded batch (default all 256; fewer for profiling)")
    ap.add_argument("--precision", type=int, default=2, choices=[0, 1, 2, 3],
                    help="Debye transform: 0 split-BF16 tensor cores, 1 FP64, 3 exact-accumulation tensor cores, "
                         "2 automatic (3 from 8e6 row x bin x q, else 1)")
    ap.add_argument("--tolerance", type=float, default=1e-4)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args, rank, world)), flush=True)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = {"cfg3": run_batch, "cfg4": run_serving, "gridexv": run_gridexv, "fit": run_fit,
            "symmetry": run_symmetry, "hydrate": run_hydrate, "atomics-peak": run_atomics_peak}.get(args.workload, run_ours)(
        args, rank, world, local_rank)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
