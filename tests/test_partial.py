"""PartialHistogramManagerMT against the reference's own partial manager over a 4-body molecule,
initially and after two rigid moves (a moved body keeps its earlier self partial; the waters belong
to body 0 and move with it, which recomputes every body-water partial and the water self partial).

CPU: the rigid moves (Body::rotate then Body::translate) reproduce the reference's coordinates, and
the combination of partial histograms (ausaxs_b200.hist.combine_partials, restated from
PartialHistogramManagerMT.cpp:152-252) over the oracle's SimpleCalculator partials reproduces the
reference's histograms.  GPU: ausaxs_b200.hist.PartialHistogramManagerMT, driven by the same moves,
over the device SimpleCalculator."""
import numpy as np
import pytest

from ausaxs_b200 import hist
from oracle import py as O
from tests.helpers import load_golden

CASE = "partial_random_4bodies"


def body_records(g, step):
    off = np.concatenate([[0], np.cumsum(g["body_sizes"])])
    xyz = g[f"coords{step}"]
    recs = np.column_stack([xyz, g["weights"]]).astype(np.float32)
    return [recs[off[k]:off[k + 1]] for k in range(len(off) - 1)]


def water_records(g, step):
    return np.column_stack([g[f"waters{step}"], g["ww"]]).astype(np.float32)


def oracle_steps(g):
    """Per step, the partials the reference holds: self partials from the first coordinates (rigid moves
    only), the cross and water partials from the current ones."""
    bw = float(g["bin_width"])
    first = body_records(g, 0)
    out = []
    for step in range(len(g["moves"]) + 1):
        cur = body_records(g, step)
        B = len(cur)
        sets = first + cur + [water_records(g, step)]
        jobs = [(k, None, 1, k) for k in range(B)] + [(2 * B, None, 1, B)]
        jobs += [(B + i, B + j, 1, i * B + j) for i in range(B) for j in range(i)]
        jobs += [(B + i, 2 * B, 1, B * B + i) for i in range(B)]
        o = O.calculator(sets, jobs, bw, 8000)
        r = hist.combine_partials([o[(0, k)] for k in range(B)], [o[(1, i * B + j)] for i in range(B) for j in range(i)],
                                  [o[(1, B * B + i)] for i in range(B)], o[(0, B)], bw)
        out.append(r)
    return out


def test_rigid_moves_match_reference():
    g = load_golden(CASE)
    off = np.concatenate([[0], np.cumsum(g["body_sizes"])])
    xyz = g["coords0"].copy()
    wat = g["waters0"].copy()
    for step, k in enumerate(g["moves"], start=1):
        R, t = g["move_R"][step - 1], g["move_t"][step - 1]
        xyz[off[k]:off[k + 1]] = hist.PartialHistogramManagerMT._rigid(xyz[off[k]:off[k + 1]], R, t)
        if k == 0:  # the waters are body 0's hydration
            wat = hist.PartialHistogramManagerMT._rigid(wat, R, t)
        np.testing.assert_allclose(xyz, g[f"coords{step}"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(wat, g[f"waters{step}"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("step", [0, 1, 2])
def test_combination_matches_reference(step):
    g = load_golden(CASE)
    r = oracle_steps(g)[step]
    assert r["max_bin"] == len(g[f"d_axis{step}"])
    for key in ("aa", "aw", "ww", "tot"):
        np.testing.assert_allclose(r[key], g[f"{key}{step}"], rtol=1e-12, atol=1e-9, err_msg=key)
    np.testing.assert_allclose(r["d_axis"], g[f"d_axis{step}"], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_device_manager_matches_reference():
    from tests.test_gpu_calc import within
    g = load_golden(CASE)
    bw = float(g["bin_width"])
    off = np.concatenate([[0], np.cumsum(g["body_sizes"])])
    bodies = [(g["coords0"][off[k]:off[k + 1]], g["weights"][off[k]:off[k + 1]]) for k in range(len(off) - 1)]
    m = hist.PartialHistogramManagerMT(bodies, (g["waters0"], g["ww"]), bw, 8000)
    wmax2 = max(float(np.max(g["weights"])), float(np.max(g["ww"]))) ** 2
    oracle = oracle_steps(g)
    for step in range(len(g["moves"]) + 1):
        if step:
            m.move_body(int(g["moves"][step - 1]), g["move_R"][step - 1], g["move_t"][step - 1])
        h = m.calculate_all()
        r = {"aa": h.get_aa_counts(), "aw": h.get_aw_counts(), "ww": h.get_ww_counts(), "tot": h.get_counts(),
             "d_axis": h.get_d_axis()}
        assert len(r["tot"]) == len(g[f"d_axis{step}"])
        # every partial carries up to (count + 1) weight-product quantisations of wmax^2 2^-30 per bin
        n_pairs = np.abs(oracle[step]["tot"]) / max(float(np.min(g["weights"])) ** 2, 1e-30) + 1
        for key in ("aa", "aw", "ww", "tot"):
            within(r[key], g[f"{key}{step}"], 4 * n_pairs * wmax2 * 2.0 ** -30 + 1e-12 * np.abs(g[f"{key}{step}"]).max(),
                   f"{key} step {step}")
        d_bound = bw * 2.0 ** -15 + (np.arange(len(r["d_axis"])) + 1) * bw * 2.0 ** -24 + 1e-9
        within(r["d_axis"], g[f"d_axis{step}"], d_bound, f"d_axis step {step}")


@pytest.mark.gpu
def test_rigid_body_step_with_regenerated_hydration():
    """One step of the reference's rigid-body loop on device entry points only: a body moves (the kept
    hydration grid loses it at its old coordinates and gets it back at the new ones), the hydration is
    regenerated, and the partial manager recomputes the moved body's cross partials and every water
    partial.  Checked against the oracle: the kept-grid hydration restatement for the waters, and its
    SimpleCalculator partials combined as the reference combines them for the histograms."""
    from ausaxs_b200 import _capi, synth
    from tests.test_gpu_calc import within

    rng = np.random.default_rng(5)
    sizes = [400, 300, 250]
    xyz = [rng.normal(c, 5.0, (n, 3)) for c, n in zip(((0, 0, 0), (16, 0, 0), (0, 17, 0)), sizes)]
    ff = [rng.choice([3, 7, 11, 12], n).astype(np.int32) for n in sizes]
    wts = [synth.ff_charge(f) for f in ff]
    allx, allf = np.concatenate(xyz), np.concatenate(ff)
    axes = O.hydrate_axes(allx)
    ctx = _capi.default_context()
    grid, ora = _capi.HydrationGrid(ctx, axes), O.HydrationGrid(axes)
    try:
        for gr in (grid, ora):
            gr.add(allx, allf)
        waters, _, _ = grid.hydrate(allx, allf)
        np.testing.assert_array_equal(waters, ora.hydrate(allx, allf)[0])
        bw = 0.25
        m = hist.PartialHistogramManagerMT(list(zip(xyz, wts)), (waters, np.full(len(waters), hist.WATER_CHARGE)), bw,
                                           8000, ctx)
        m.calculate_all()
        first = [np.column_stack([x, w]).astype(np.float32) for x, w in zip(xyz, wts)]
        # move body 1 about its centre, as the rigid-body transforms do
        k, ang = 1, 0.3
        R = np.array([[np.cos(ang), -np.sin(ang), 0], [np.sin(ang), np.cos(ang), 0], [0, 0, 1]])
        c = xyz[k].mean(0)
        new = (xyz[k] - c) @ R.T + c + np.array([1.5, -2.0, 0.7])
        for gr in (grid, ora):
            gr.remove(xyz[k], ff[k])
            gr.add(new, ff[k])
        xyz[k] = new
        order = [0, 2, 1]  # the re-added body comes last in the grid's member list
        members, types = np.concatenate([xyz[b] for b in order]), np.concatenate([ff[b] for b in order])
        waters2, _, _ = grid.hydrate(members, types)
        np.testing.assert_array_equal(waters2, ora.hydrate(members, types)[0])
        m.set_body_coordinates(k, new)
        m.set_waters(waters2, np.full(len(waters2), hist.WATER_CHARGE))
        h = m.calculate_all()
    finally:
        grid.close()
    B = len(sizes)
    cur = [np.column_stack([x, w]).astype(np.float32) for x, w in zip(xyz, wts)]
    wrec = np.column_stack([waters2, np.full(len(waters2), hist.WATER_CHARGE)]).astype(np.float32)
    jobs = [(b, None, 1, b) for b in range(B)] + [(2 * B, None, 1, B)]
    jobs += [(B + i, B + j, 1, i * B + j) for i in range(B) for j in range(i)]
    jobs += [(B + i, 2 * B, 1, B * B + i) for i in range(B)]
    o = O.calculator(first + cur + [wrec], jobs, bw, 8000)
    ref = hist.combine_partials([o[(0, b)] for b in range(B)], [o[(1, i * B + j)] for i in range(B) for j in range(i)],
                                [o[(1, B * B + i)] for i in range(B)], o[(0, B)], bw)
    got = {"aa": h.get_aa_counts(), "aw": h.get_aw_counts(), "ww": h.get_ww_counts(), "tot": h.get_counts(),
           "d_axis": h.get_d_axis()}
    assert len(got["tot"]) == ref["max_bin"]
    wmax2 = max(float(np.max(np.concatenate(wts))), hist.WATER_CHARGE) ** 2
    n_pairs = np.abs(ref["tot"]) / min(float(np.min(np.concatenate(wts))), hist.WATER_CHARGE) ** 2 + 1
    for key in ("aa", "aw", "ww", "tot"):
        within(got[key], ref[key], 4 * n_pairs * wmax2 * 2.0 ** -30 + 1e-12 * np.abs(ref[key]).max(), key)
    within(got["d_axis"], ref["d_axis"], bw * 2.0 ** -15 + (np.arange(len(ref["d_axis"])) + 1) * bw * 2.0 ** -24 + 1e-9,
           "d_axis")
