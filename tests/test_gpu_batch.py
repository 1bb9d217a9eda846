"""Batched profiles (many structures, one captured graph) against the single-structure path and the
oracle.  The batch shares launches but not accumulators, and everything before the FP64 transform is
integer arithmetic, so each structure's histograms are identical to its single-structure ones and
its I(q) equal to the last bit."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist, synth
from oracle import py as O

pytestmark = pytest.mark.gpu


def _molecules(seed, sizes, waters=0.2, exv=0):
    out = []
    for k, n in enumerate(sizes):
        rng = np.random.default_rng(seed + k)
        xyz = rng.normal(0, 3.0 * max(n, 1) ** (1 / 3), (n, 3))
        ff = rng.choice([3, 7, 11, 12], n, p=[0.63, 0.17, 0.19, 0.01]).astype(np.int32)
        nw = int(round(waters * n))
        wat = rng.normal(0, 3.6 * max(n, 1) ** (1 / 3), (nw, 3))
        x = np.round(rng.uniform(-6, 6, (exv, 3))) if exv else None
        out.append(hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, exv=x, volume=18.0 * max(n, 1)))
    return out


SIZES = [1, 2, 7, 130, 257, 900, 2600, 4099, 513, 64, 3000, 11000]


def test_batch_equals_single_structure_ffavg(gpu_ctx):
    mols = _molecules(100, SIZES)
    q = np.linspace(0.005, 0.8, 400)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    I = B.debye_transform(q, cw=1.1, cx=0.95)
    for i, m in enumerate(mols):
        ref = hist.profile(hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx), q, cw=1.1, cx=0.95)
        np.testing.assert_allclose(I[i], ref, rtol=1e-13, atol=0, err_msg=f"structure {i} ({len(m.atoms)} atoms)")
        h = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
        b = B.histogram(i)
        assert b["max_bin"] == h.max_bin
        np.testing.assert_array_equal(b["aa"], h.get_raw_aa_counts_by_ff())
        np.testing.assert_array_equal(b["aw"], h.get_raw_aw_counts_by_ff())
        np.testing.assert_array_equal(b["d_axis"], h.get_d_axis())
    B.close()


@pytest.mark.parametrize("precision", [1, 2])
def test_batch_vs_oracle(gpu_ctx, precision):
    """FP64 transform (1) and the exact-accumulation tensor-core transform (2) against the oracle."""
    mols = _molecules(7, [300, 1200, 50, 2500])
    q = np.linspace(0.005, 0.5, 120)
    I = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx).debye_transform(q, precision=precision)
    for i, m in enumerate(mols):
        A, W, _ = m.compact_ff()
        o = O.hist_ff(0, A, W, None, 0.25, 8000, m.volume * 0.334 / m.size_atom())
        Io, _ = O.debye_ff(0, o, q)
        np.testing.assert_allclose(I[i], Io, rtol=1e-6)


def test_batch_ffgrid_equals_single_structure(gpu_ctx):
    mols = _molecules(40, [400, 1500, 90], exv=700)
    q = np.linspace(0.01, 1.0, 150)
    I = hist.BatchedProfiles(mols, grid=True, bin_width=0.1, ctx=gpu_ctx).debye_transform(q, cw=0.9, cx=1.05)
    for i, m in enumerate(mols):
        ref = hist.profile(hist.HistogramManagerMTFFGrid(m, 0.1, 8000, gpu_ctx), q, cw=0.9, cx=1.05)
        np.testing.assert_allclose(I[i], ref, rtol=1e-13, atol=0)


def test_autotune_candidates_agree_and_graph_replays(gpu_ctx):
    mols = _molecules(9, [20000, 700, 3000, 150, 9000])
    q = np.linspace(0.005, 0.8, 200)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    I0 = B.debye_transform(q)
    choice, times = B.autotune()
    assert 0 <= choice < 7 and np.all(times[:7] > 0)
    assert _capi.Batch.candidate(choice)["tile_small"] in (256, 512)
    I1 = B.debye_transform(q)        # new plan: graph captured again
    I2 = B.debye_transform(q)        # replay
    np.testing.assert_array_equal(I0, I1)
    np.testing.assert_array_equal(I1, I2)
    I3 = B.debye_transform(q[:50])   # new q: captured again
    np.testing.assert_array_equal(I3, I0[:, :50])
    B.close()


def test_batch_rejects_simple_manager(gpu_ctx):
    cfg = _capi.HistConfig(_capi.MANAGER_MT, 1, 0.25, 8000, 0.0)
    a = np.zeros((3, 4), np.float32)
    with pytest.raises(_capi.AusaxsError):
        _capi.Batch(gpu_ctx, cfg, [a], [np.zeros((0, 4), np.float32)])


def _moved(mols, seed, scale=0.97, jitter=0.05, volume_scale=0.9):
    """Same atoms (types, order) and waters in new positions: a rotation about the centroid, a
    shrink (pair distances stay inside the bins planned for the originals) and a small jitter."""
    rng = np.random.default_rng(seed)
    out = []
    for m in mols:
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        c = m.atoms.mean(axis=0) if len(m.atoms) else np.zeros(3)
        mv = lambda p: (((p - c) @ q.T) * scale + c + rng.uniform(-jitter, jitter, p.shape)) if len(p) else p
        out.append(hist.Molecule(atoms=mv(m.atoms), ff_types=m.ff_types.copy(), waters=mv(m.waters),
                                 volume=m.volume * volume_scale))
    return out


def test_set_points_equals_a_new_batch(gpu_ctx):
    mols = _molecules(300, SIZES)
    q = np.linspace(0.005, 0.8, 400)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    I0 = B.debye_transform(q, cw=1.1, cx=0.95)
    for k in range(2):  # two successive replacements, each a replay of the same graph
        new = _moved(mols, 77 + k)
        B.set_molecules(new)
        I = B.debye_transform(q, cw=1.1, cx=0.95)
        F = hist.BatchedProfiles(new, bin_width=0.25, ctx=gpu_ctx)
        If = F.debye_transform(q, cw=1.1, cx=0.95)
        np.testing.assert_allclose(I, If, rtol=1e-13, atol=0)
        for i in range(len(new)):
            b, f = B.histogram(i), F.histogram(i)
            assert b["max_bin"] == f["max_bin"]
            np.testing.assert_array_equal(b["aa"], f["aa"])
            np.testing.assert_array_equal(b["aw"], f["aw"])
            np.testing.assert_array_equal(b["ww"], f["ww"])
            np.testing.assert_array_equal(b["d_axis"], f["d_axis"])
        F.close()
        assert np.max(np.abs(I / I0 - 1)) > 1e-6  # the profiles did change
    # and against the oracle for the small ones
    for i, m in enumerate(new[:6]):
        A, W, _ = m.compact_ff()
        o = O.hist_ff(0, A, W, None, 0.25, 8000, m.volume * 0.334 / m.size_atom())
        Io, _ = O.debye_ff(0, o, q, cw=1.1, cx=0.95)
        np.testing.assert_allclose(I[i], Io, rtol=1e-6)
    B.close()


def test_set_points_rejections_and_recovery(gpu_ctx):
    mols = _molecules(500, [400, 1300, 90])
    q = np.linspace(0.005, 0.5, 100)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    I0 = B.debye_transform(q)
    parts = [m.compact_ff() for m in mols]
    atoms = [p[0].copy() for p in parts]
    waters = [p[1].copy() for p in parts]
    bad = [a.copy() for a in atoms]
    t = bad[1][5, 3].view(np.int32)
    bad[1][5, 3] = np.array([3 if t != 3 else 7], np.int32).view(np.float32)[0]  # another form-factor type
    with pytest.raises(_capi.AusaxsError) as e:
        B._b.set_points(bad, waters)
    assert e.value.code == _capi.ERR_ARGUMENT
    with pytest.raises(_capi.AusaxsError) as e:  # every profile fails until valid points arrive
        B.debye_transform(q)
    assert e.value.code == _capi.ERR_ARGUMENT
    wbad = [w.copy() for w in waters]
    wbad[0][3, 1] = np.nan
    with pytest.raises(_capi.AusaxsError):
        B._b.set_points(atoms, wbad)
    B._b.set_points(atoms, waters)
    np.testing.assert_array_equal(B.debye_transform(q), I0)
    # a structure grown beyond the bins planned for it: bin overflow, then recovery
    grown = [a.copy() for a in atoms]
    grown[2][:, :3] *= 3.0
    B._b.set_points(grown, waters)
    with pytest.raises(_capi.AusaxsError) as e:
        B.debye_transform(q)
    assert e.value.code == _capi.ERR_BIN_OVERFLOW
    B._b.set_points(atoms, waters)
    np.testing.assert_array_equal(B.debye_transform(q), I0)
    with pytest.raises(_capi.AusaxsError):
        B._b.set_points(atoms[:2], waters)  # not the creation shapes
    B.close()


def test_set_points_device_arrays(gpu_ctx):
    import torch

    mols = _molecules(600, [700, 2100])
    q = np.linspace(0.005, 0.5, 100)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    B.debye_transform(q)
    new = _moved(mols, 5, volume_scale=1.0)
    parts = [m.compact_ff() for m in new]
    a = torch.from_numpy(np.concatenate([p[0] for p in parts])).cuda()
    w = torch.from_numpy(np.concatenate([p[1] for p in parts])).cuda()
    torch.cuda.synchronize()
    B._b.set_points_device(a, w)
    I = B.debye_transform(q)
    If = hist.BatchedProfiles(new, bin_width=0.25, ctx=gpu_ctx).debye_transform(q)
    np.testing.assert_allclose(I, If, rtol=1e-13, atol=0)
    B.close()


@pytest.mark.parametrize("grid", [False, True])
def test_batch_tensor_core_transform_within_tolerance(gpu_ctx, grid):
    """The exact-accumulation tensor-core transform (int8 digit products of the histogram rows and of
    shared Taylor tables, s32 sums) against the FP64 transform of the same histograms: within the
    tolerance wherever it keeps its own value, equal wherever it fell back."""
    sizes = [300, 2600, 40, 9000, 1200, 700] if not grid else [400, 1500, 90]
    mols = _molecules(800, sizes, exv=700 if grid else 0)
    w = 0.1 if grid else 0.25
    q = np.linspace(0.005, 1.0 if grid else 0.8, 333)
    B = hist.BatchedProfiles(mols, grid=grid, bin_width=w, ctx=gpu_ctx)
    I64 = B.debye_transform(q, cw=1.1, cx=0.95)
    Itc = B.debye_transform(q, cw=1.1, cx=0.95, precision=2, tolerance=1e-4)
    fell_back = B.fp64_columns()
    rel = np.abs(Itc / I64 - 1)
    assert np.max(rel) <= 1e-4, float(np.max(rel))
    # the bound is rigorous and tight enough that almost every value stays on the tensor cores
    assert fell_back <= 0.05 * Itc.size, fell_back
    # the actual deviation is far below the tolerance (integer sums, 42-bit digits, 2^-32 truncation)
    assert np.median(rel) < 1e-8, float(np.median(rel))
    # a tolerance nothing meets: every value recomputed in FP64, identical to the FP64 transform
    Iall = B.debye_transform(q, cw=1.1, cx=0.95, precision=2, tolerance=1e-300)
    assert B.fp64_columns() == Itc.size
    np.testing.assert_array_equal(Iall, I64)
    B.close()


def test_batch_tensor_core_transform_after_set_points(gpu_ctx):
    mols = _molecules(900, [500, 3000, 150])
    q = np.linspace(0.005, 0.8, 200)
    B = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx)
    B.debye_transform(q, precision=2)
    new = _moved(mols, 3)
    B.set_molecules(new)
    Itc = B.debye_transform(q, precision=2)
    I64 = hist.BatchedProfiles(new, bin_width=0.25, ctx=gpu_ctx).debye_transform(q)
    assert np.max(np.abs(Itc / I64 - 1)) <= 1e-4
    B.close()
