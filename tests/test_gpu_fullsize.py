"""Full-size configurations, checked through properties that do not need the oracle (which cannot
finish these sizes in seconds): pair-count conservation per histogram block, distance-axis
consistency (every weighted bin mean lies inside its bin), and the tensor-core transform against
the FP64 transform within the path's I(q) bar (1e-4 relative)."""
import numpy as np
import pytest

from ausaxs_b200 import hist, synth

pytestmark = pytest.mark.gpu


def _check_axis(d, width):
    b = np.arange(len(d))
    # bin b holds distances d with rint(d / width) = b: its mean is within half a bin of b * width
    # (float rounding of d / width allows 1e-6 relative more); bin 0 is pinned to 0
    assert d[0] == 0
    assert np.all(np.abs(d[1:] - b[1:] * width) <= 0.5 * width * (1 + 1e-6) + 1e-6 * d[1:])


def _tc_vs_fp64(h, q):
    h.precision, h.tolerance = 1, 1e-5
    _, I64 = h.debye_transform(q)
    h.precision, h.tolerance = 0, 1e-4
    _, Itc = h.debye_transform(q)
    np.testing.assert_allclose(Itc, I64, rtol=1e-4, atol=0)


def test_cfg1_grid_counts_and_transform(gpu_ctx):
    w = synth.cfg1()
    m = w.molecules[0]
    na, nw, nx = m.size_atom(), m.size_water(), len(m.exv)
    h = hist.HistogramManagerMTFFGrid(m, w.bin_width, w.bin_count, gpu_ctx).calculate_all()
    aa, aw, ww = h.get_raw_aa_counts_by_ff(), h.get_raw_aw_counts_by_ff(), h.get_raw_ww_counts_by_ff()
    assert aa[1:, 1:].sum() == na * na          # 2 x pairs + self terms
    assert aa[1:, 0].sum() == na * nx           # atom-dummy cross (factor 1)
    assert aa[0, 0].sum() == nx * nx            # dummy-dummy
    assert aw[1:].sum() == na * nw and aw[0].sum() == nw * nx
    assert ww.sum() == nw * nw
    _check_axis(h.get_d_axis(), w.bin_width)
    _tc_vs_fp64(h, w.q)


def test_cfg2_icosahedral_shell(gpu_ctx):
    w = synth.cfg2()
    m = w.molecules[0]
    na, nw = m.size_atom(), m.size_water()
    h = hist.HistogramManagerMTFFAvg(m, True, w.bin_width, w.bin_count, gpu_ctx).calculate_all()
    aa, aw, ww = h.get_raw_aa_counts_by_ff(), h.get_raw_aw_counts_by_ff(), h.get_raw_ww_counts_by_ff()
    assert aa[1:, 1:].sum() == na * na
    assert aw[1:].sum() == na * nw
    assert ww.sum() == nw * nw
    assert h.get_counts().sum() == na * na + na * nw + nw * nw
    assert h.max_bin > 2500  # the 150 A shell spans about 3,000 bins of 0.1 A
    _check_axis(h.get_d_axis(), w.bin_width)
    _tc_vs_fp64(h, w.q)
