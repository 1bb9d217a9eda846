"""The oracle (oracle/oracle.c) pinned against the reference's outputs and known answers.

CPU only.  The golden fixtures under tests/golden/ were produced by the reference compiled from
its own sources (tests/golden/make_golden.py); when that build is present here
(oracle/_ref/libausaxs_ref.so) the oracle is also compared with it on fresh random inputs.
"""
import numpy as np
import pytest

from oracle import py as O
from tests.helpers import FIT_KIND, calc_cases, calc_inputs, fit_cases, grid_cases, golden_cases, load_golden, oracle_for

CASES = golden_cases()


def test_fixtures_present():
    assert len(CASES) >= 15


@pytest.mark.parametrize("name", CASES)
def test_oracle_histograms_match_reference(name):
    g = load_golden(name)
    o = oracle_for(g)
    mb = len(g["d_axis"])
    assert len(o.d_axis) == mb, "max_bin truncation differs"
    assert o.overflow == 0
    if str(g["manager"]) == "mt":
        # weighted counts: FP64 sums of float weight products (order-only differences)
        np.testing.assert_allclose(o.aa, g["aa"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(o.aw, g["aw"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(o.ww, g["ww_h"], rtol=1e-12, atol=1e-9)
    else:
        # integer pair counts: exact
        np.testing.assert_array_equal(o.aa, g["aa"])
        np.testing.assert_array_equal(o.aw, g["aw"])
        np.testing.assert_array_equal(o.ww, g["ww_h"])
        if "d_axis_ax" in g:
            np.testing.assert_allclose(o.d_axis_ax, g["d_axis_ax"], rtol=0, atol=1e-9)
            np.testing.assert_allclose(o.d_axis_xx, g["d_axis_xx"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(o.d_axis, g["d_axis"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("name", CASES)
def test_oracle_intensity_matches_reference(name):
    g = load_golden(name)
    o = oracle_for(g)
    cw, cx, crho, dwa, dwx = g["params"]
    q = g["q"]
    if str(g["manager"]) == "mt":
        I = O.debye_simple(o, q, cw)
        np.testing.assert_allclose(I, g["Iq"], rtol=1e-10)
        return
    kind = {"ffavg": 0, "ffexplicit": 1, "ffgrid": 2}[str(g["manager"])]
    I, prof = O.debye_ff(kind, o, q, cw, cx, crho, dwa, dwx)
    scale = np.abs(g["Iq"]).max()
    np.testing.assert_allclose(I, g["Iq"], rtol=1e-9, atol=1e-12 * scale)
    for k in range(6):
        ref = g["profiles"][k]
        np.testing.assert_allclose(prof[k], ref, rtol=1e-9, atol=1e-12 * max(np.abs(ref).max(), 1.0))


def test_simple_cube_known_answer():
    """SimpleCube: 8 corners and a centre; distances 9x0, 16xsqrt3, 24x2, 24xsqrt8, 8xsqrt12
    (tests/feature/hist/hist_test_helper.h:87-162 of the reference)."""
    g = load_golden("cube_mt")
    atoms = g["atoms"]
    A = O.pack_points(atoms, np.ones(len(atoms)), False)
    W = O.pack_points(np.zeros((0, 3)), np.zeros(0), False)
    h = O.hist_simple(A, W, 0.25, 8000)
    want = np.zeros(len(h.aa))
    for d, n in [(0, 9), (np.sqrt(3), 16), (2, 24), (np.sqrt(8), 24), (np.sqrt(12), 8)]:
        want[int(np.rint(np.float32(d) * 4))] += n
    np.testing.assert_array_equal(h.aa, want)


def test_linear_lsq_known_answer():
    x = np.linspace(1, 10, 40)
    y = 2.5 * x + 0.75
    a, b, _, _, chi2 = O.linear_lsq(x, y, np.ones_like(x))
    assert abs(a - 2.5) < 1e-12 and abs(b - 0.75) < 1e-11 and chi2 < 1e-20


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_reference_fresh_random():
    rng = np.random.default_rng(7)
    na, nw = 611, 133
    xyz = rng.normal(0, 9, (na, 3))
    ff = rng.choice([3, 7, 11, 12], na)
    wat = rng.normal(0, 11, (nw, 3))
    O.ref_set_axes(0.25, 8000, 1e-4, 0.5)
    O.ref_set_simple_exv(False)
    m = O.RefMolecule(xyz, np.ones(na), ff, wat, np.ones(nw), volume=3000.0)
    m.set_manager("ffavg")
    h = m.calculate()
    aa, aw, ww = h.ff()
    o = O.hist_ff(0, O.pack_points(xyz, ff, True), O.pack_points(wat, np.ones(nw, np.int32), True), None, 0.25, 8000,
                  3000.0 * 0.334 / na)
    np.testing.assert_array_equal(o.aa, aa)
    np.testing.assert_array_equal(o.aw, aw)
    np.testing.assert_array_equal(o.ww, ww)


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
def test_linear_lsq_matches_reference():
    rng = np.random.default_rng(3)
    x = rng.uniform(1, 100, 50)
    y = 0.3 * x + 4 + rng.normal(0, 1, 50)
    e = rng.uniform(0.5, 2, 50)
    r = O.ref_linear_lsq(x, y, e)
    o = O.linear_lsq(x, y, e)
    np.testing.assert_allclose(o[[0, 1, 4]], r[[0, 1, 4]], rtol=1e-10)


@pytest.mark.parametrize("name", grid_cases())
def test_oracle_grid_exv_matches_reference(name):
    g = load_golden(name)
    d, vol = O.grid_exv(g["atoms"], g["ff"], g["waters"])
    np.testing.assert_array_equal(d, g["dummies"])  # same cells, same (x-major) order
    assert vol == float(g["volume"]) == len(d)


@pytest.mark.parametrize("name", fit_cases())
def test_oracle_fit_matches_reference(name):
    """SmartFitter::fit (Golden over one parameter): the same search path, so the same parameter value
    and evaluation count; a, b and chi2 to rounding."""
    g = load_golden(name)
    kind = FIT_KIND[str(g["manager"])]
    v, a, b, chi2, n = O.fit(kind, oracle_for(g), g["q"], g["y"], g["sigma"], int(g["fit_param"]), base=g["fit_base"])
    r = g["fit_out"]
    assert v == r[0] and n == int(r[4])
    np.testing.assert_allclose([a, b, chi2], r[1:4], rtol=1e-10)


@pytest.mark.parametrize("name", calc_cases())
def test_oracle_calculator_matches_reference(name):
    """SimpleCalculator jobs with scaling factors and merge ids: values, counts and bin-centre sums exact."""
    g = load_golden(name)
    sets, jobs = calc_inputs(g)
    o = O.calculator(sets, jobs, float(g["bin_width"]), 8000)
    assert sorted(o) == [tuple(k) for k in g["keys"]]
    for r, k in enumerate(g["keys"]):
        n = g["results"].shape[2]
        for i in range(3):
            np.testing.assert_array_equal(o[tuple(k)][i][:n], g["results"][r][i])
            assert not np.any(o[tuple(k)][i][n:])
