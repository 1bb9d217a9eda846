"""Excluded-volume dummies of the molecular grid on the device (RawGridExv on the expanded grid)
against the reference's fixtures and the oracle, and the FFGrid / FFAvg paths that take their
excluded volume from that grid.  Bar: the same cells in the same order, the same volume, integer
counts bit-identical to those built from the oracle's dummies, and I(q) within 1e-5 relative."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist
from oracle import py as O
from tests.helpers import grid_cases, load_golden

pytestmark = pytest.mark.gpu


def _records(xyz, ff):
    return hist.pack(xyz, ff, True)


@pytest.mark.parametrize("name", grid_cases())
def test_grid_dummies_vs_reference(name, gpu_ctx):
    g = load_golden(name)
    a = _records(g["atoms"], g["ff"])
    w = _records(g["waters"], np.ones(len(g["waters"]), np.int32))
    d, vol = _capi.grid_exv(gpu_ctx, a, w)
    np.testing.assert_array_equal(d[:, :3], g["dummies"].astype(np.float32))
    assert np.all(d[:, 3].view(np.int32) == 0)  # form_factor_t EXCLUDED_VOLUME
    assert vol == float(g["volume"])


@pytest.mark.parametrize("seed,na,nw,spread", [(1, 1, 0, 5.0), (2, 40, 0, 3.0), (3, 2000, 400, 12.0), (4, 6000, 0, 30.0)])
def test_grid_dummies_vs_oracle(seed, na, nw, spread, gpu_ctx):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(0, spread, (na, 3)).astype(np.float32).astype(np.float64)
    ff = rng.choice(np.arange(1, 15), na).astype(np.int32)
    wat = rng.normal(0, spread * 1.2, (nw, 3)).astype(np.float32).astype(np.float64)
    d, vol = _capi.grid_exv(gpu_ctx, _records(xyz, ff), _records(wat, np.ones(nw, np.int32)))
    do, vo = O.grid_exv(xyz, ff, wat)
    np.testing.assert_array_equal(d[:, :3].astype(np.float64), do)
    assert vol == vo


def test_ffgrid_from_grid_equals_given_dummies(gpu_ctx):
    rng = np.random.default_rng(5)
    xyz = rng.normal(0, 10, (1800, 3)).astype(np.float32).astype(np.float64)
    ff = rng.choice([3, 4, 5, 7, 8, 11, 12], 1800).astype(np.int32)
    wat = rng.normal(0, 12, (300, 3)).astype(np.float32).astype(np.float64)
    dummies, _ = O.grid_exv(xyz, ff, wat)
    m_grid = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, volume=1.0)           # dummies from the grid
    m_given = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat, exv=dummies, volume=1.0)
    h1 = hist.HistogramManagerMTFFGrid(m_grid, 0.1, 8000, gpu_ctx).calculate_all()
    h2 = hist.HistogramManagerMTFFGrid(m_given, 0.1, 8000, gpu_ctx).calculate_all()
    np.testing.assert_array_equal(h1.get_raw_aa_counts_by_ff(), h2.get_raw_aa_counts_by_ff())
    np.testing.assert_array_equal(h1.get_raw_aw_counts_by_ff(), h2.get_raw_aw_counts_by_ff())
    np.testing.assert_array_equal(h1.get_d_axis_xx(), h2.get_d_axis_xx())
    o = O.hist_ff(2, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(len(wat), np.int32), True),
                  O.pack_points(dummies, np.zeros(len(dummies), np.int32), True), 0.1, 8000, 0.0)
    np.testing.assert_array_equal(h1.get_raw_aa_counts_by_ff(), o.aa)
    q = np.linspace(0.01, 0.8, 120)
    I = hist.profile(hist.HistogramManagerMTFFGrid(m_grid, 0.1, 8000, gpu_ctx), q)
    # the transform alone: the oracle's FP64 Debye sum over the device's own histogram
    own = O.FFHist(h1.get_raw_aa_counts_by_ff(), h1.get_raw_aw_counts_by_ff(), h1.get_raw_ww_counts_by_ff(),
                   h1.get_counts(), h1.get_d_axis(), h1.get_d_axis_ax(), h1.get_d_axis_xx())
    np.testing.assert_allclose(I, O.debye_ff(2, own, q)[0], rtol=1e-9)
    # end to end: the weighted bin centres differ from the oracle's by at most a few 1e-7 A
    # (fixed-point residuals), which moves the high-q tail by a few 1e-6 relative; bound 1e-5
    Io, _ = O.debye_ff(2, o, q)
    np.testing.assert_allclose(I, Io, rtol=1e-5)


def test_ffavg_z_from_grid_volume(gpu_ctx):
    rng = np.random.default_rng(6)
    xyz = rng.normal(0, 9, (1200, 3)).astype(np.float32).astype(np.float64)
    ff = rng.choice([3, 7, 11, 12], 1200).astype(np.int32)
    wat = rng.normal(0, 11, (200, 3)).astype(np.float32).astype(np.float64)
    _, vol = O.grid_exv(xyz, ff, wat)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=wat)  # no volume: Molecule::get_volume_grid()
    assert m.get_volume_grid() == vol
    h = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx).calculate_all()
    o = O.hist_ff(0, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(len(wat), np.int32), True), None,
                  0.25, 8000, vol * 0.334 / len(xyz))
    np.testing.assert_array_equal(h.get_raw_aa_counts_by_ff(), o.aa)
    q = np.linspace(0.005, 0.5, 100)
    _, I = h.debye_transform(q)
    Io, _ = O.debye_ff(0, o, q)
    np.testing.assert_allclose(I, Io, rtol=1e-5)


def test_grid_dummies_device_pointers_and_capacity(gpu_ctx):
    import torch

    g = load_golden("gridexv_random1")
    a = _records(g["atoms"], g["ff"])
    w = _records(g["waters"], np.ones(len(g["waters"]), np.int32))
    dev = torch.device("cuda:0")
    a_d, w_d = torch.from_numpy(a).to(dev), torch.from_numpy(w).to(dev)
    n_ref = len(g["dummies"])
    small = torch.zeros((n_ref - 1, 4), dtype=torch.float32, device=dev)
    out = torch.zeros((n_ref, 4), dtype=torch.float32, device=dev)
    torch.cuda.synchronize()  # the library runs on its context's stream
    with pytest.raises(_capi.AusaxsError) as e:
        _capi.grid_exv_device(gpu_ctx, a_d, len(a), w_d, len(w), small, n_ref - 1)
    assert e.value.code == _capi.ERR_CAPACITY
    n, vol = _capi.grid_exv_device(gpu_ctx, a_d, len(a), w_d, len(w), out, n_ref)
    assert n == n_ref and vol == float(g["volume"])
    np.testing.assert_array_equal(out.cpu().numpy()[:, :3], g["dummies"].astype(np.float32))
    # no atoms: an empty grid, volume 0
    n0, v0 = _capi.grid_exv_device(gpu_ctx, a_d, 0, w_d, len(w), out, n_ref)
    assert n0 == 0 and v0 == 0.0


def test_structure_from_grid_equals_given_dummies(gpu_ctx):
    import torch

    rng = np.random.default_rng(7)
    xyz = rng.normal(0, 11, (2500, 3)).astype(np.float32).astype(np.float64)
    ff = rng.choice([3, 4, 5, 7, 8, 11, 12], 2500).astype(np.int32)
    wat = rng.normal(0, 13, (400, 3)).astype(np.float32).astype(np.float64)
    a, w = _records(xyz, ff), _records(wat, np.ones(len(wat), np.int32))
    d, _ = _capi.grid_exv(gpu_ctx, a, w)
    cfg = _capi.HistConfig(_capi.MANAGER_FFGRID, 1, 0.1, 8000, 0.0)
    params = _capi.DebyeParams(1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5)
    q = torch.linspace(0.01, 0.6, 90, dtype=torch.float64, device="cuda:0")
    out = []
    for st in (_capi.Structure(gpu_ctx, a, w, exv_from_grid=True), _capi.Structure(gpu_ctx, a, w, exv=d)):
        I = torch.zeros(90, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        st.profile_device(cfg, q, 90, params, I)
        torch.cuda.synchronize()
        out.append(I.cpu().numpy())
        st.close()
    np.testing.assert_array_equal(out[0], out[1])
    with pytest.raises(_capi.AusaxsError):  # grid dummies need form-factor types
        _capi.Structure(gpu_ctx, a, w, ff_typed=False, exv_from_grid=True)


def test_grid_dummies_edge_cases(gpu_ctx):
    """Waters only (no atoms: nothing is kept) and a single atom of each van der Waals radius class."""
    w = _records(np.array([[0.0, 0.0, 0.0], [5.0, 1.0, -2.0]]), np.ones(2, np.int32))
    d, vol = _capi.grid_exv(gpu_ctx, np.zeros((0, 4), np.float32), w)
    assert len(d) == 0 and vol == 0.0
    for ff in (2, 3, 7, 11, 12, 14):
        xyz = np.array([[0.3, -0.2, 0.7]])
        d, vol = _capi.grid_exv(gpu_ctx, _records(xyz, np.array([ff], np.int32)), np.zeros((0, 4), np.float32))
        do, vo = O.grid_exv(xyz.astype(np.float32).astype(np.float64), np.array([ff]), None)
        np.testing.assert_array_equal(d[:, :3].astype(np.float64), do)
        assert vol == vo
