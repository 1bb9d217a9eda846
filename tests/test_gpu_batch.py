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


def test_batch_vs_oracle(gpu_ctx):
    mols = _molecules(7, [300, 1200, 50])
    q = np.linspace(0.005, 0.5, 120)
    I = hist.BatchedProfiles(mols, bin_width=0.25, ctx=gpu_ctx).debye_transform(q)
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
