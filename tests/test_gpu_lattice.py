"""Grid dummies' self pairs by the lattice kernel (occupancy autocorrelation) against the oracle's
pair-by-pair evaluation.

Dummies on integer or half-integer coordinates of a 1 A lattice take the lattice path (checked through
the context's kernel timing: class 6 launches); at 0.1 A bins some integer squared distances are exact
rounding ties, where the reference's scalar-tail pairs (last row length mod 4 partners of each row)
round away from zero, so the tail correction is exercised too.  Bar: counts bit-exact, distance axes
within bin_width * 2^-15, exactly as the pair kernel."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist
from oracle import py as O

pytestmark = pytest.mark.gpu


def d_atol(bw):
    return bw * 2.0 ** -15


def _ball_lattice(seed, radius, offset):
    rng = np.random.default_rng(seed)
    r = int(np.ceil(radius))
    g = np.stack(np.meshgrid(*[np.arange(-r, r + 1)] * 3, indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    g = g[(g ** 2).sum(1) <= radius ** 2]
    g = g[rng.random(len(g)) < 0.9]  # holes
    g = g[rng.permutation(len(g))]   # the reference's order is the caller's
    return g + offset


@pytest.mark.parametrize("offset,bw,nx_extra", [(0.0, 0.1, 0), (0.5, 0.1, 1), (0.5, 0.25, 2), (0.0, 0.25, 3)])
def test_lattice_self_pairs_vs_oracle(offset, bw, nx_extra, gpu_ctx):
    rng = np.random.default_rng(7 + nx_extra)
    exv = _ball_lattice(11 + nx_extra, 11.0, offset)[: 4000 + nx_extra]  # ragged tails: n mod 4 varies
    xyz = rng.normal(0, 6, (700, 3))
    ff = rng.choice([3, 7, 11, 12], len(xyz), p=[0.63, 0.17, 0.19, 0.01]).astype(np.int32)
    wat = rng.normal(0, 9, (150, 3))
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, exv=exv, volume=1.0)
    ctx = _capi.Context(0)
    ctx.enable_timing(True)
    h = hist.HistogramManagerMTFFGrid(m, bw, 8000, ctx).calculate_all()
    _, launches = ctx.kernel_time(6)
    ctx.enable_timing(False)
    assert launches >= 1, "the lattice path was not taken"
    o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(len(wat), np.int32), True),
                  O.pack_points(exv, np.zeros(len(exv), np.int32), True), bw, 8000, 0.0)
    assert h.max_bin == len(o.d_axis)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), o.aw)
    np.testing.assert_allclose(h.get_d_axis_xx(), o.d_axis_xx, atol=d_atol(bw), rtol=0)
    np.testing.assert_allclose(h.get_d_axis_ax(), o.d_axis_ax, atol=d_atol(bw), rtol=0)
    np.testing.assert_allclose(h.get_d_axis(), o.d_axis, atol=d_atol(bw), rtol=0)
    ctx.close()


def _tie_lattice(seed, offset):
    """A sparse lattice spanning ~130 A whose last point has many partners at squared distances that
    are exact rounding ties at 0.1 A bins (x = d * float(1 / 0.1) a half-integer): the last point is a
    scalar-tail partner of three rows in four, so the tail correction has pairs to move."""
    inv_w = np.float32(1 / 0.1)
    s2 = np.arange(1, 3 * 99 ** 2, dtype=np.float32)
    x = np.sqrt(s2) * inv_w
    ties = s2[(x - np.floor(x)) == 0.5].astype(int)
    assert len(ties) > 0
    rng = np.random.default_rng(seed)
    last = np.array([99, 99, 99])
    pts = {tuple(int(v) for v in rng.integers(0, 100, 3)) for _ in range(1500)}
    rngv = np.arange(0, 100)
    for t in ties[:6]:
        for a in rngv:
            for b in rngv:
                c2 = t - a * a - b * b
                if c2 < 0:
                    continue
                c = int(round(np.sqrt(c2)))
                if c * c == c2 and c < 100 and rng.random() < 0.5:
                    pts.add((int(last[0] - a), int(last[1] - b), int(last[2] - c)))
    pts.discard(tuple(last))
    arr = np.array(sorted(pts), np.float64)
    arr = arr[rng.permutation(len(arr))]
    return np.vstack([arr, last[None, :].astype(np.float64)]) + offset


@pytest.mark.parametrize("offset", [0.0, 0.5])
def test_lattice_rounding_ties_vs_oracle(offset, gpu_ctx):
    exv = _tie_lattice(19, offset)
    rng = np.random.default_rng(2)
    xyz = rng.uniform(0, 99, (200, 3))
    ff = np.full(len(xyz), 3, np.int32)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=np.zeros((0, 3)), exv=exv, volume=1.0)
    ctx = _capi.Context(0)
    ctx.enable_timing(True)
    h = hist.HistogramManagerMTFFGrid(m, 0.1, 8000, ctx).calculate_all()
    _, launches = ctx.kernel_time(6)
    ctx.enable_timing(False)
    assert launches >= 1, "the lattice path was not taken"
    o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(np.zeros((0, 3)), np.zeros(0, np.int32), True),
                  O.pack_points(exv, np.zeros(len(exv), np.int32), True), 0.1, 8000, 0.0)
    assert h.max_bin == len(o.d_axis)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_allclose(h.get_d_axis_xx(), o.d_axis_xx, atol=d_atol(0.1), rtol=0)
    ctx.close()


def test_off_lattice_dummies_use_the_pair_kernel(gpu_ctx):
    rng = np.random.default_rng(3)
    exv = _ball_lattice(5, 10.0, 0.0)[:2000] + np.array([0.25, 0.0, 0.0])  # quarter offsets: not eligible
    xyz = rng.normal(0, 6, (300, 3))
    ff = np.full(len(xyz), 3, np.int32)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=np.zeros((0, 3)), exv=exv, volume=1.0)
    ctx = _capi.Context(0)
    ctx.enable_timing(True)
    h = hist.HistogramManagerMTFFGrid(m, 0.1, 8000, ctx).calculate_all()
    _, launches = ctx.kernel_time(6)
    ctx.enable_timing(False)
    assert launches == 0
    o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(np.zeros((0, 3)), np.zeros(0, np.int32), True),
                  O.pack_points(exv, np.zeros(len(exv), np.int32), True), 0.1, 8000, 0.0)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    ctx.close()


def test_reloaded_dummies_are_not_binned_with_a_stale_lattice(gpu_ctx):
    """One-shot calls reuse the context's scratch structure: after a lattice-eligible set of dummies,
    a set of the same size with two dummies in one cell (not eligible) and then an eligible set with
    other positions must each match the oracle (the lattice and the plan built for the previous
    points are discarded on reload)."""
    rng = np.random.default_rng(29)
    xyz = rng.normal(0, 6, (400, 3))
    ff = np.full(len(xyz), 3, np.int32)
    n = 3000
    base = _ball_lattice(31, 10.0, 0.0)[:n]
    dup = base.copy()
    dup[-1] = dup[0]                              # shared cell
    moved = _ball_lattice(37, 10.0, 0.5)[:n]      # other positions, half-integer
    for exv in (base, dup, moved, base):
        m = hist.Molecule(atoms=xyz, ff_types=ff, waters=np.zeros((0, 3)), exv=exv, volume=1.0)
        h = hist.HistogramManagerMTFFGrid(m, 0.1, 8000, gpu_ctx).calculate_all()
        o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(np.zeros((0, 3)), np.zeros(0, np.int32), True),
                      O.pack_points(exv, np.zeros(len(exv), np.int32), True), 0.1, 8000, 0.0)
        assert h.max_bin == len(o.d_axis)
        np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
        np.testing.assert_allclose(h.get_d_axis_xx(), o.d_axis_xx, atol=d_atol(0.1), rtol=0)
