"""Rigid-body serving: incremental inter-body recompute against a full recompute of the moved
assembly, results alone vs mixed with other requests, admission by footprint and slots.

Bar: exact.  Every pair keeps the full assembly's loop geometry and all accumulation is integer, so
the master histogram after any sequence of moves equals HistogramManagerMTFFAvg::calculate_all() of
the moved coordinates bit for bit, and I(q) equals the single-structure transform of it."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist, synth
from oracle import py as O

pytestmark = pytest.mark.gpu

RHO = 0.334


def _bodies(seed, sizes, waters=0.15):
    rng = np.random.default_rng(seed)
    atoms, wats, ffs = [], [], []
    for k, n in enumerate(sizes):
        xyz, ff = synth.globule(seed * 10 + k, n)
        xyz = xyz + rng.uniform(-25, 25, 3)
        nw = int(round(waters * n))
        w = synth.waters(seed * 10 + k + 5, xyz, ff, nw) if nw else np.zeros((0, 3))
        atoms.append(hist.pack(xyz, ff, True))
        wats.append(hist.pack(w, np.ones(len(w), np.int32), True))
        ffs.append(ff)
    return atoms, wats, ffs


def _cfg(atoms, volume_per_atom=18.0):
    n = sum(len(a) for a in atoms)
    return _capi.HistConfig(_capi.MANAGER_FFAVG, 1, 0.25, 8000, volume_per_atom * n * RHO / n)


def _random_move(rng, center, max_deg=5.0, max_t=2.0):
    R = synth.random_rotation(rng, max_deg)
    t = rng.uniform(-1, 1, 3)
    t *= max_t * rng.uniform() / max(np.linalg.norm(t), 1e-12)
    # rotation about the body's centroid: x <- R (x - c) + c + t
    return R, center - R @ center + t


def _full(server, sid, ffs, cfg, q, gpu_ctx):
    a, w = server.coordinates(sid)
    m = hist.Molecule(atoms=a[:, :3].astype(np.float64), ff_types=np.concatenate(ffs),
                      waters=w[:, :3].astype(np.float64), volume=cfg.z_exv * len(a) / RHO)
    mgr = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx)
    return mgr.calculate_all(), hist.profile(mgr, q)


def test_moves_equal_full_recompute(gpu_ctx):
    atoms, wats, ffs = _bodies(3, [700, 1500, 400, 1100])
    cfg = _cfg(atoms)
    q = np.linspace(0.005, 0.5, 120)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    S = _capi.Server(hbm_budget=2 << 30)
    sid, fp = S.admit(cfg, atoms, wats, q, p, margin=30.0)
    assert fp > 0
    rng = np.random.default_rng(1)
    for step in range(6):
        body = int(rng.integers(0, 4)) if step else -1
        if body >= 0:
            R, t = _random_move(rng, S.body_center(sid, body), max_deg=20.0, max_t=4.0)
            tk = S.submit(sid, body, R, t)
        else:
            tk = S.submit(sid)
        I, fit = S.wait(tk, sid)
        h, I_full = _full(S, sid, ffs, cfg, q, gpu_ctx)
        g = S.histogram(sid, 8000)
        assert g["max_bin"] == h.max_bin
        np.testing.assert_array_equal(g["aa"], h.get_raw_aa_counts_by_ff())
        np.testing.assert_array_equal(g["aw"], h.get_raw_aw_counts_by_ff())
        np.testing.assert_array_equal(g["ww"], h.get_raw_ww_counts_by_ff())
        np.testing.assert_array_equal(g["d_axis"], h.get_d_axis())
        np.testing.assert_allclose(I, I_full, rtol=1e-13, atol=0)
    S.close()


def test_alone_equals_mixed(gpu_ctx):
    atoms, wats, _ = _bodies(5, [900, 600, 1300])
    others = [_bodies(s, [800, 1000, 500]) for s in (6, 7)]
    q = np.linspace(0.005, 0.5, 100)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    rng = np.random.default_rng(2)
    moves = [(int(rng.integers(0, 3)), synth.random_rotation(rng, 5.0), rng.uniform(-2, 2, 3)) for _ in range(8)]

    S1 = _capi.Server(hbm_budget=2 << 30)
    a_id, _ = S1.admit(_cfg(atoms), atoms, wats, q, p)
    alone = [S1.wait(S1.submit(a_id, b, R, t), a_id)[0] for b, R, t in moves]
    S1.close()

    # the same moves with two other assemblies' moves in flight around each of them, and every
    # move of this assembly submitted before any of its results is read
    mixed = []
    S3 = _capi.Server(hbm_budget=2 << 30, slots_per_assembly=8)
    ids = [S3.admit(_cfg(o[0]), o[0], o[1], q, p)[0] for o in others]
    a3, _ = S3.admit(_cfg(atoms), atoms, wats, q, p)
    rng = np.random.default_rng(9)
    pending = []
    for b, R, t in moves:
        other_tk = [(oid, S3.submit(oid, int(rng.integers(0, 3)), synth.random_rotation(rng, 5.0),
                                    rng.uniform(-2, 2, 3))) for oid in ids]
        tk = S3.submit(a3, b, R, t)
        pending.append(tk)
        for oid, otk in other_tk:
            S3.wait(otk, oid)
    for tk in pending:
        mixed.append(S3.wait(tk, a3)[0])
    S3.close()
    for x, y in zip(alone, mixed):
        np.testing.assert_array_equal(x, y)


def test_fit_matches_oracle_lsq(gpu_ctx):
    atoms, wats, _ = _bodies(11, [600, 800])
    q = np.linspace(0.005, 0.5, 80)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    S = _capi.Server(hbm_budget=1 << 30)
    sid, _ = S.admit(_cfg(atoms), atoms, wats, q, p)
    I0, _ = S.wait(S.submit(sid), sid)
    rng = np.random.default_rng(3)
    target = I0 * 1.7 + 5.0 + rng.normal(0, 0.01 * np.abs(I0))
    err = 0.01 * np.abs(I0)
    S.close()
    S = _capi.Server(hbm_budget=1 << 30)
    sid, _ = S.admit(_cfg(atoms), atoms, wats, q, p, target=target, target_err=err)
    I1, fit = S.wait(S.submit(sid, 1, synth.random_rotation(rng, 5.0), np.array([0.5, -0.3, 1.0])), sid)
    ref = O.linear_lsq(target, I1, err)  # {a, b, var_a, var_b, chi2}; the device returns sigmas
    np.testing.assert_allclose(fit[[0, 1, 4]], ref[[0, 1, 4]], rtol=1e-9)
    np.testing.assert_allclose(fit[[2, 3]], np.sqrt(ref[[2, 3]]), rtol=1e-9)
    S.close()


def test_admission_by_footprint_and_slots(gpu_ctx):
    atoms, wats, _ = _bodies(13, [500, 700])
    q = np.linspace(0.005, 0.5, 50)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    probe = _capi.Server(hbm_budget=1 << 40)
    _, fp = probe.admit(_cfg(atoms), atoms, wats, q, p)
    probe.close()
    S = _capi.Server(hbm_budget=int(fp * 1.5), max_inflight=64, slots_per_assembly=2)
    a, _ = S.admit(_cfg(atoms), atoms, wats, q, p)
    with pytest.raises(_capi.AusaxsError) as e:
        S.admit(_cfg(atoms), atoms, wats, q, p)
    assert e.value.code == _capi.ERR_CAPACITY
    used, budget, _ = S.usage()
    assert used == fp and budget == int(fp * 1.5)
    t1, t2 = S.submit(a), S.submit(a)
    assert S.try_submit(a) is None  # both slots in flight
    S.wait(t1, a)
    t3 = S.submit(a)
    S.wait(t2, a)
    S.wait(t3, a)
    with pytest.raises(_capi.AusaxsError) as e:
        S.wait(t3, a)
    assert e.value.code == _capi.ERR_NOT_FOUND
    S.release(a)
    b, _ = S.admit(_cfg(atoms), atoms, wats, q, p)
    assert S.usage()[0] == fp
    S.close()


def test_wait_times_out_then_completes(gpu_ctx):
    """ausaxs_gpu_server_wait's bound: a zero timeout on a request that is still on the GPU gives
    AUSAXS_ERR_TIMEOUT and leaves the ticket in flight; a normal wait then returns the result, equal
    to the other requests'.  Four full recomputes of a ~56k-atom assembly (several milliseconds of pair
    work each) are queued before the zero-timeout wait on the last one; should the host fall behind
    the GPU that long, the round is repeated (up to five times)."""
    atoms, wats, _ = _bodies(17, [20000, 15000, 12000, 9000])
    q = np.linspace(0.005, 0.5, 60)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    S = _capi.Server(hbm_budget=4 << 30, slots_per_assembly=4)
    sid, _ = S.admit(_cfg(atoms), atoms, wats, q, p)
    timed_out = False
    for _ in range(5):
        tickets = [S.submit(sid) for _ in range(4)]
        last = None
        try:
            last = S.wait(tickets[-1], sid, timeout_ms=0)
        except _capi.AusaxsError as e:
            assert e.code == _capi.ERR_TIMEOUT
            timed_out = True
        Is = [S.wait(t, sid)[0] for t in tickets[:-1]]
        Is.append(last[0] if last is not None else S.wait(tickets[-1], sid)[0])
        for I in Is[1:]:
            np.testing.assert_array_equal(I, Is[0])
        if timed_out:
            break
    assert timed_out
    S.close()


def test_served_iq_matches_oracle_after_moves(gpu_ctx):
    """An 8-body assembly shaped like the serving configuration (bodies of 300-1200 atoms, waters on
    every body): after each of 4 random rigid moves the served I(q) equals the oracle's FP64 profile
    of the moved coordinates (HistogramManagerMTFFAvg + the generalised-q transform), not only the
    device's own full recompute."""
    rng = np.random.default_rng(41)
    sizes = [int(x) for x in np.exp(rng.uniform(np.log(300), np.log(1200), 8))]
    atoms, wats, ffs = _bodies(23, sizes, waters=0.1)
    cfg = _cfg(atoms)
    q = np.linspace(0.005, 0.5, 400)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    S = _capi.Server(hbm_budget=2 << 30)
    sid, _ = S.admit(cfg, atoms, wats, q, p, margin=30.0)
    ff = np.concatenate(ffs).astype(np.int32)
    for step in range(4):
        body = int(rng.integers(0, 8))
        R, t = _random_move(rng, S.body_center(sid, body))
        I, _ = S.wait(S.submit(sid, body, R, t), sid)
        a, w = S.coordinates(sid)
        o = O.hist_ff(0, O.pack_points(a[:, :3].astype(np.float64), ff, True),
                      O.pack_points(w[:, :3].astype(np.float64), np.ones(len(w), np.int32), True), None, 0.25, 8000,
                      cfg.z_exv)
        Io, _ = O.debye_ff(0, o, q)
        # the d-axis carries the fixed-point quantisation (<= 1e-6 A): q * 1e-6 relative phase at most
        np.testing.assert_allclose(I, Io, rtol=1e-6, atol=0)
    S.close()


def test_served_tensor_core_transform(gpu_ctx):
    """Requests of an assembly admitted with precision 3 (the exact-accumulation tensor-core transform,
    its tables kept with the assembly) against the same moves served with the FP64 transform: within
    the 1e-4 bar, and the assembly's histograms identical."""
    atoms, wats, _ = _bodies(11, [1200, 2500, 800, 1700])
    cfg = _cfg(atoms)
    q = np.linspace(0.005, 0.5, 400)
    p64 = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    ptc = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 3, 1e-4)
    S = _capi.Server(hbm_budget=4 << 30)
    a, _ = S.admit(cfg, atoms, wats, q, p64, margin=30.0)
    b, _ = S.admit(cfg, atoms, wats, q, ptc, margin=30.0)
    rng = np.random.default_rng(4)
    for step in range(5):
        body = int(rng.integers(0, 4))
        R, t = _random_move(rng, S.body_center(a, body))
        Ia, _ = S.wait(S.submit(a, body, R, t), a)
        Ib, _ = S.wait(S.submit(b, body, R, t), b)
        np.testing.assert_allclose(Ib, Ia, rtol=1e-4, atol=0)
        np.testing.assert_array_equal(S.histogram(a, 8000)["aa"], S.histogram(b, 8000)["aa"])
    S.close()


def test_submission_order_policy_same_results(gpu_ctx):
    """Scheduling changes when a request runs, not what it computes: the same moves under both policies
    give the same bits."""
    atoms, wats, _ = _bodies(13, [900, 1400, 600])
    others = _bodies(14, [700, 1100])
    q = np.linspace(0.005, 0.5, 100)
    p = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    rng = np.random.default_rng(5)
    moves = [(int(rng.integers(0, 3)), synth.random_rotation(rng, 5.0), rng.uniform(-2, 2, 3)) for _ in range(6)]
    results = []
    for policy in (0, 1, 2):
        S = _capi.Server(hbm_budget=2 << 30)
        S.set_policy(policy)
        a, _ = S.admit(_cfg(atoms), atoms, wats, q, p)
        b, _ = S.admit(_cfg(others[0]), others[0], others[1], q, p)
        out = []
        for body, R, t in moves:
            ta = S.submit(a, body, R, t)
            tb = S.submit(b, body % 2, R, t)  # interleaved with another assembly's requests
            out.append(S.wait(ta, a)[0])
            S.wait(tb, b)
        results.append(np.array(out))
        S.close()
    np.testing.assert_array_equal(results[0], results[1])
    np.testing.assert_array_equal(results[0], results[2])
    with pytest.raises(_capi.AusaxsError):
        _capi.Server(hbm_budget=1 << 30).set_policy(-1)
