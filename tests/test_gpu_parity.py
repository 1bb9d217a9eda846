"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's golden outputs.

Bar: pair counts bit-exact; weighted counts and distance axes within the fixed-point resolution of
the on-chip accumulators (stated per assertion); I(q) within 1e-9 relative of the FP64 oracle
(the FP64 transform path).
"""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist, synth
from oracle import py as O
from tests.helpers import golden_cases, load_golden, oracle_for, simple_exv_weights

pytestmark = pytest.mark.gpu

# d-axis: the in-bin offset of every pair is quantised to about c * 2^-15 (c = bin width), so a bin
# mean is within c * 2^-16 of the FP64 mean (<= 3.8e-6 A at 0.25 A bins, 1.5e-6 A at 0.1 A); the
# tolerance is twice that bound.
def d_atol(bin_width):
    return bin_width * 2.0 ** -15


D_ATOL = d_atol(0.25)
# weighted counts: weight products quantised to 2^-k with max|w|^2 * 2^k <= 2^30
W_RTOL = 1e-7


def molecule_from_golden(g):
    w = g["w"]
    if str(g["manager"]) == "mt" and bool(g["simple_exv"]):
        w = simple_exv_weights(w, float(g["volume"]), len(g["atoms"]))
    return hist.Molecule(atoms=g["atoms"], ff_types=g["ff"], weights=w, waters=g["waters"], water_weights=g["ww"],
                         exv=g["exv"], volume=float(g["volume"]))


def manager_for(g, ctx):
    m = molecule_from_golden(g)
    bw = float(g["bin_width"])
    mgr = str(g["manager"])
    if mgr == "mt":
        return hist.HistogramManagerMT(m, True, bw, 8000, ctx)
    if mgr == "ffavg":
        return hist.HistogramManagerMTFFAvg(m, True, bw, 8000, ctx)
    if mgr == "ffexplicit":
        return hist.HistogramManagerMTFFExplicit(m, True, bw, 8000, ctx)
    return hist.HistogramManagerMTFFGrid(m, bw, 8000, ctx)


@pytest.mark.parametrize("name", golden_cases())
def test_histograms_vs_reference_golden(name, gpu_ctx):
    g = load_golden(name)
    h = manager_for(g, gpu_ctx).calculate_all()
    mb = len(g["d_axis"])
    assert h.max_bin == mb
    if str(g["manager"]) == "mt":
        np.testing.assert_allclose(h.get_aa_counts(), g["aa"], rtol=W_RTOL, atol=1e-6)
        np.testing.assert_allclose(h.get_aw_counts(), g["aw"], rtol=W_RTOL, atol=1e-6)
        np.testing.assert_allclose(h.get_ww_counts(), g["ww_h"], rtol=W_RTOL, atol=1e-6)
    else:
        np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), g["aa"])
        np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), g["aw"])
        np.testing.assert_array_equal(h.get_raw_ww_counts_by_ff(), g["ww_h"])
        if "d_axis_ax" in g:
            np.testing.assert_allclose(h.get_d_axis_ax(), g["d_axis_ax"], atol=d_atol(float(g["bin_width"])), rtol=0)
            np.testing.assert_allclose(h.get_d_axis_xx(), g["d_axis_xx"], atol=d_atol(float(g["bin_width"])), rtol=0)
    np.testing.assert_allclose(h.get_d_axis(), g["d_axis"], atol=d_atol(float(g["bin_width"])), rtol=0)


@pytest.mark.parametrize("name", golden_cases())
def test_intensity_vs_reference_golden(name, gpu_ctx):
    g = load_golden(name)
    h = manager_for(g, gpu_ctx).calculate_all()
    cw, cx, crho, dwa, dwx = g["params"]
    h.apply_water_scaling_factor(cw)
    if str(g["manager"]) != "mt":
        h.apply_excluded_volume_scaling_factor(cx)
        h.apply_solvent_density_scaling_factor(crho)
        h.apply_atomic_debye_waller_factor(dwa)
        h.apply_exv_debye_waller_factor(dwx)
    q, I = h.debye_transform(g["q"])
    # the d-axis carries the fixed-point quantisation (<= 1e-6 A): q * 1e-6 relative phase at most
    np.testing.assert_allclose(I, g["Iq"], rtol=1e-6)
    prof = h.profiles(g["q"])
    for k in range(6):
        ref = g["profiles"][k]
        np.testing.assert_allclose(prof[k], ref, rtol=1e-6, atol=1e-9 * max(np.abs(ref).max(), 1.0))


def _random_ff(seed, na, nw, nx=0, spread=12.0):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(0, spread, (na, 3))
    ff = rng.choice([3, 7, 11, 12], na, p=[0.63, 0.17, 0.19, 0.01]).astype(np.int32)
    wat = rng.normal(0, spread * 1.2, (nw, 3))
    exv = np.round(rng.uniform(-spread, spread, (nx, 3)))
    return xyz, ff, wat, exv


@pytest.mark.parametrize("na,nw,bw", [(1, 0, 0.25), (2, 1, 0.25), (5, 3, 0.25), (257, 31, 0.25), (1024, 256, 0.25),
                                      (1031, 257, 0.1), (3000, 600, 0.25), (4099, 0, 0.1)])
def test_ffavg_vs_oracle_ragged(na, nw, bw, gpu_ctx):
    xyz, ff, wat, _ = _random_ff(na * 7 + nw, na, nw)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=20.0 * na)
    h = hist.HistogramManagerMTFFAvg(m, True, bw, 8000, gpu_ctx).calculate_all()
    o = O.hist_ff(0, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(nw, np.int32), True), None, bw, 8000,
                  20.0 * na * 0.334 / na)
    assert h.max_bin == len(o.d_axis)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), o.aw)
    np.testing.assert_array_equal(h.get_raw_ww_counts_by_ff(), o.ww)
    np.testing.assert_allclose(h.get_d_axis(), o.d_axis, atol=d_atol(bw), rtol=0)


def test_ffgrid_vs_oracle(gpu_ctx):
    xyz, ff, wat, exv = _random_ff(5, 2000, 400, 3000)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, exv=exv, volume=1.0)
    h = hist.HistogramManagerMTFFGrid(m, 0.1, 8000, gpu_ctx).calculate_all()
    o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(len(wat), np.int32), True),
                  O.pack_points(exv, np.zeros(len(exv), np.int32), True), 0.1, 8000, 0.0)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), o.aw)
    np.testing.assert_allclose(h.get_d_axis_ax(), o.d_axis_ax, atol=d_atol(0.1), rtol=0)
    np.testing.assert_allclose(h.get_d_axis_xx(), o.d_axis_xx, atol=d_atol(0.1), rtol=0)
    q = np.linspace(0.005, 1.0, 300)
    I, prof = hist.profile(hist.HistogramManagerMTFFGrid(m, 0.1, 8000, gpu_ctx), q, cw=1.1, cx=0.9,
                           with_profiles=True)
    Io, po = O.debye_ff(2, o, q, 1.1, 0.9)
    np.testing.assert_allclose(I, Io, rtol=1e-6, atol=1e-9 * np.abs(Io).max())


@pytest.mark.parametrize("manager,na,nw,nx", [("ffavg", 3000, 600, 0), ("ffgrid", 2000, 400, 16500)])
def test_wide_histograms_vs_oracle(manager, na, nw, nx, gpu_ctx):
    """About 3,000 bins of 0.1 A with 16 type-pair rows: the u64 offset sums move to registers so every
    row stays on chip (256-point tiles for the FFAvg case, 512-point tiles for the FFGrid case, which
    has more than 16,384 dummies)."""
    xyz, ff, wat, exv = _random_ff(17 + na, na, nw, nx, spread=30.0)
    kind = {"ffavg": 0, "ffgrid": 2}[manager]
    if kind == 2:
        m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, exv=exv, volume=1.0)
        h = hist.HistogramManagerMTFFGrid(m, 0.1, 8000, gpu_ctx).calculate_all()
    else:
        m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=20.0 * na)
        h = hist.HistogramManagerMTFFAvg(m, True, 0.1, 8000, gpu_ctx).calculate_all()
    o = O.hist_ff(kind, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(nw, np.int32), True),
                  O.pack_points(exv, np.zeros(nx, np.int32), True) if nx else None, 0.1, 8000,
                  0.0 if kind == 2 else 20.0 * na * 0.334 / na)
    assert h.max_bin == len(o.d_axis) and 1500 < h.max_bin < 3300  # 16 rows fit on chip only with register sums
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), o.aw)
    np.testing.assert_array_equal(h.get_raw_ww_counts_by_ff(), o.ww)
    np.testing.assert_allclose(h.get_d_axis(), o.d_axis, atol=d_atol(0.1), rtol=0)
    if kind == 2:
        np.testing.assert_allclose(h.get_d_axis_ax(), o.d_axis_ax, atol=d_atol(0.1), rtol=0)
        np.testing.assert_allclose(h.get_d_axis_xx(), o.d_axis_xx, atol=d_atol(0.1), rtol=0)


def test_ffexplicit_vs_oracle(gpu_ctx):
    xyz, ff, wat, _ = _random_ff(21, 2200, 500)
    ff[::37] = 14  # some OTHER atoms (argon excluded volume)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=1.0)
    h = hist.HistogramManagerMTFFExplicit(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    o = O.hist_ff(1, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(len(wat), np.int32), True), None,
                  0.25, 8000, 0.0)
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    q = np.linspace(0.005, 0.8, 250)
    h.apply_water_scaling_factor(1.07)
    h.apply_excluded_volume_scaling_factor(1.04)
    h.apply_solvent_density_scaling_factor(0.98)
    h.apply_atomic_debye_waller_factor(0.3)
    _, I = h.debye_transform(q)
    Io, po = O.debye_ff(1, o, q, 1.07, 1.04, 0.98, 0.3, 0.0)
    np.testing.assert_allclose(I, Io, rtol=1e-6, atol=1e-9 * np.abs(Io).max())
    prof = h.profiles(q)
    for k in range(6):
        np.testing.assert_allclose(prof[k], po[k], rtol=1e-6, atol=1e-9 * max(np.abs(po[k]).max(), 1.0))


def test_mt_vs_oracle(gpu_ctx):
    rng = np.random.default_rng(11)
    xyz = rng.normal(0, 10, (2500, 3))
    w = rng.uniform(-0.5, 9.0, 2500)  # implicit excluded volume can make weights small or negative
    wat = rng.normal(0, 12, (500, 3))
    ww = np.full(500, 9.0)
    m = hist.Molecule(atoms=xyz, weights=w, waters=wat, water_weights=ww)
    h = hist.HistogramManagerMT(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    o = O.hist_simple(O.pack_points(xyz, w, False), O.pack_points(wat, ww, False), 0.25, 8000)
    assert h.max_bin == len(o.d_axis)
    scale = np.abs(o.aa).max()
    np.testing.assert_allclose(h.get_aa_counts(), o.aa, rtol=W_RTOL, atol=1e-9 * scale)
    np.testing.assert_allclose(h.get_aw_counts(), o.aw, rtol=W_RTOL, atol=1e-9 * scale)
    np.testing.assert_allclose(h.get_ww_counts(), o.ww, rtol=W_RTOL, atol=1e-9 * scale)
    np.testing.assert_allclose(h.get_d_axis(), o.d_axis, atol=D_ATOL, rtol=0)
    q = np.linspace(0.005, 0.5, 100)
    _, I = h.debye_transform(q)
    np.testing.assert_allclose(I, O.debye_simple(o, q), rtol=1e-6)


def test_profile_fused_equals_two_step(gpu_ctx):
    w = synth.cfg0()
    m = w.molecules[0]
    mgr = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx)
    h = mgr.calculate_all()
    _, I2 = h.debye_transform(w.q)
    I1 = hist.profile(mgr, w.q)
    np.testing.assert_allclose(I1, I2, rtol=1e-12)


def test_cfg0_vs_oracle(gpu_ctx):
    w = synth.cfg0()
    m = w.molecules[0]
    h = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    A, W, _ = m.compact_ff()
    o = O.hist_ff(0, A, W, None, 0.25, 8000, m.volume * 0.334 / m.size_atom())
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    np.testing.assert_array_equal(h.get_raw_aw_counts_by_ff(), o.aw)
    np.testing.assert_allclose(h.get_d_axis(), o.d_axis, atol=D_ATOL, rtol=0)
    _, I = h.debye_transform(w.q)
    Io, _ = O.debye_ff(0, o, w.q)
    np.testing.assert_allclose(I, Io, rtol=1e-6)


def test_linear_lsq_vs_oracle(gpu_ctx):
    rng = np.random.default_rng(4)
    n = 400
    target = 1e4 * np.exp(-np.linspace(0.005, 0.5, n) * 20)
    err = 0.01 * target
    model = 3.2 * target + 7.0 + rng.normal(0, 1, n) * err
    g = _capi.linear_lsq(gpu_ctx, target, model, err)
    o = O.linear_lsq(target, model, err)
    np.testing.assert_allclose(g[[0, 1, 4]], o[[0, 1, 4]], rtol=1e-9)
    np.testing.assert_allclose(g[[2, 3]], np.sqrt(o[[2, 3]]), rtol=1e-9)


# ---- error behaviour -----------------------------------------------------------------------

def test_unknown_form_factor_is_an_error(gpu_ctx):
    xyz, ff, wat, _ = _random_ff(1, 50, 5)
    ff[7] = 16  # form_factor_t::UNKNOWN
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=1.0)
    with pytest.raises(_capi.AusaxsError) as e:
        hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    assert e.value.code == _capi.ERR_FORM_FACTOR


def test_bin_overflow_is_an_error(gpu_ctx):
    xyz, ff, wat, _ = _random_ff(2, 100, 10, spread=30.0)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=1.0)
    with pytest.raises(_capi.AusaxsError) as e:
        hist.HistogramManagerMTFFAvg(m, True, 0.25, 50, gpu_ctx).calculate_all()
    assert e.value.code == _capi.ERR_BIN_OVERFLOW


def test_non_finite_coordinates_are_an_error(gpu_ctx):
    xyz, ff, wat, _ = _random_ff(3, 60, 6)
    xyz[3, 1] = np.nan
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=1.0)
    with pytest.raises(_capi.AusaxsError) as e:
        hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    assert e.value.code == _capi.ERR_ARGUMENT


def test_all_pairs_in_one_bin(gpu_ctx):
    """Atomic contention stress: every pair lands in bin 0 (coincident atoms)."""
    n = 3000
    xyz = np.zeros((n, 3))
    ff = np.full(n, 3, np.int32)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=np.zeros((0, 3)), volume=1.0)
    h = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    aa = h.get_raw_aa_counts_by_ff()
    assert aa[3, 3, 0] == n * (n - 1) + n
    rest = aa.copy()
    rest[3, 3, 0] = rest[3, 0, 0] = rest[0, 0, 0] = 0
    assert not rest.any()
    z = 1.0 * 0.334 / n
    assert aa[3, 0, 0] == n * (n - 1) * z
    assert aa[0, 0, 0] == (n * (n - 1) + n) * (z * z)
