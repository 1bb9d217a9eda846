"""The device fit (SmartFitter with the Golden minimiser over one parameter) against the reference's
own fits and the oracle.

Bar: the same parameter value as the reference to within the search tolerance (1e-4; the chi2 sums
are reduced in a different order, so a comparison between two nearly equal trial values may go the
other way), the same number of evaluations when the value is the same, chi2, a and b within 1e-6
relative."""
import numpy as np
import pytest

from ausaxs_b200 import _capi, hist
from ausaxs_b200.fitter import SmartFitter
from oracle import py as O
from tests.helpers import FIT_KIND, fit_cases, load_golden, oracle_for
from tests.test_gpu_parity import manager_for

pytestmark = pytest.mark.gpu
PARAMS = ("cw", "cx", "crho", "dw_atomic", "dw_exv")


@pytest.mark.parametrize("name", fit_cases())
def test_fit_vs_reference(name, gpu_ctx):
    g = load_golden(name)
    h = manager_for(g, gpu_ctx).calculate_all()
    r = SmartFitter((g["q"], g["y"], g["sigma"]), h).fit(PARAMS[int(g["fit_param"])])
    ref = g["fit_out"]
    assert abs(r.value - ref[0]) <= 1e-4
    if r.value == ref[0]:
        assert r.evaluations == int(ref[4])
    np.testing.assert_allclose([r.a, r.b, r.chi2], ref[1:4], rtol=1e-6)
    # the fitted curve is the linear fit of the model at the fitted value
    assert np.sum(((g["y"] - r.I_fit) / g["sigma"]) ** 2) == pytest.approx(r.chi2, rel=1e-9)


@pytest.mark.parametrize("param,limits,tol", [("cw", (0.5, 3.0), 1e-6), ("crho", None, 1e-3), ("dw_exv", (0.0, 2.0), 1e-5),
                                              ("cx", (1.0, 1.0 + 5e-5), 1e-4)])
def test_fit_options_vs_oracle(param, limits, tol, gpu_ctx):
    g = load_golden("fit_random_ffavg_cw")
    m = manager_for(g, gpu_ctx)
    h = m.calculate_all()
    h.apply_solvent_density_scaling_factor(1.05)  # a non-default value of a parameter that is not fitted
    k = PARAMS.index(param)
    r = SmartFitter((g["q"], g["y"], g["sigma"]), h).fit(param, limits, tol)
    base = [1.0, 1.0, 1.05, 0.0, 0.0]
    lo, hi = limits if limits is not None else O.FIT_LIMITS[k]
    oh = oracle_for(g)
    o = O.fit(FIT_KIND["ffavg"], oh, g["q"], g["y"], g["sigma"], k, lo, hi, tol, base)
    # the device histogram's weighted bin centres differ from the oracle's at the fixed-point level, which
    # can move the chi2 minimum by about 1e-6: compare the searches to the larger of that and tol, and
    # the linear fit at the device's own value (an interval of width 0 is not searched)
    assert abs(r.value - o[0]) <= max(tol, 4e-6)
    at = O.fit(FIT_KIND["ffavg"], oh, g["q"], g["y"], g["sigma"], k, r.value, r.value, tol, base)
    assert at[0] == r.value and at[4] == 0
    np.testing.assert_allclose([r.a, r.b, r.chi2], at[1:4], rtol=1e-6)
    if limits is not None and limits[1] - limits[0] < tol:  # no search: the centre of the interval
        assert r.value == limits[0] + (limits[1] - limits[0]) / 2 and r.evaluations == 0


def test_structure_fit_equals_host_fit(gpu_ctx):
    import torch

    g = load_golden("fit_random_ffgrid_cx")
    m = manager_for(g, gpu_ctx)
    h = m.calculate_all()
    host = SmartFitter((g["q"], g["y"], g["sigma"]), h).fit("cx")
    a, w, x = m._inputs()
    st = _capi.Structure(gpu_ctx, a, w, x)
    dev = torch.device("cuda:0")
    q, y, s = (torch.from_numpy(np.ascontiguousarray(v)).to(dev) for v in (g["q"], g["y"], g["sigma"]))
    I_fit = torch.zeros(len(g["q"]), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    r = st.fit_device(m.config(), q, y, s, len(g["q"]), _capi.DebyeParams(1, 1, 1, 0, 0, 1, 1, 0),
                      _capi.FitOptions(1, 0, 0, 1e-4), I_fit)
    st.close()
    assert r.value == host.value and r.evaluations == host.evaluations
    np.testing.assert_allclose([r.a, r.b, r.chi2], [host.a, host.b, host.chi2], rtol=1e-12)
    np.testing.assert_allclose(I_fit.cpu().numpy(), host.I_fit, rtol=1e-12)


def test_fit_argument_errors(gpu_ctx):
    g = load_golden("fit_random_mt_cw")
    h = manager_for(g, gpu_ctx).calculate_all()
    with pytest.raises(_capi.AusaxsError):  # the Simple histogram has the water scaling only
        SmartFitter((g["q"], g["y"], g["sigma"]), h).fit("cx")
    with pytest.raises(ValueError):
        SmartFitter((g["q"], g["y"][:-1], g["sigma"]), h)


def test_fit_minimum_outside_the_interval(gpu_ctx):
    """The Golden search converges to the interval's edge when the minimum lies beyond it, as the
    reference does; the oracle takes the same path."""
    g = load_golden("fit_random_ffavg_cw")  # truth cw = 1.6
    h = manager_for(g, gpu_ctx).calculate_all()
    r = SmartFitter((g["q"], g["y"], g["sigma"]), h).fit("cw", (2.0, 4.0))
    o = O.fit(FIT_KIND["ffavg"], oracle_for(g), g["q"], g["y"], g["sigma"], 0, 2.0, 4.0)
    assert abs(r.value - 2.0) < 1e-4 and abs(r.value - o[0]) <= 1e-4


@pytest.mark.parametrize("param", ["dw_atomic", "dw_exv"])
def test_fit_debye_waller_vs_oracle(param, gpu_ctx):
    g = load_golden("fit_random_ffavg_dwa")
    h = manager_for(g, gpu_ctx).calculate_all()
    k = PARAMS.index(param)
    r = SmartFitter((g["q"], g["y"], g["sigma"]), h).fit(param)
    o = O.fit(FIT_KIND["ffavg"], oracle_for(g), g["q"], g["y"], g["sigma"], k)
    assert abs(r.value - o[0]) <= 1e-4
    np.testing.assert_allclose(r.chi2, o[3], rtol=1e-6)
