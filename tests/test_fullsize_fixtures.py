"""The full-size fixtures (reference output for the benchmark configurations) are self-consistent and
their inputs regenerate from the seeds.  CPU only: the GPU comparison is tests/test_gpu_fullsize.py."""
import numpy as np
import pytest

from ausaxs_b200 import synth
from oracle import py as O
from tests.helpers import input_digest, load_golden


def _ffhist(g, suffix=""):
    ax = g.get("d_axis_ax" + suffix)
    xx = g.get("d_axis_xx" + suffix)
    return O.FFHist(np.asarray(g["aa" + suffix], np.float64), np.asarray(g["aw" + suffix], np.float64),
                    np.asarray(g["ww_h" + suffix], np.float64), g["tot" + suffix], g["d_axis" + suffix], ax, xx)


@pytest.mark.parametrize("name,gen,kind", [("fullsize_cfg1", synth.cfg1, 2), ("fullsize_cfg2", synth.cfg2, 0)])
def test_single_structure_fixture(name, gen, kind):
    g = load_golden(name)
    w = gen()
    m = w.molecules[0]
    assert input_digest(m) == str(g["digest"])
    na, nw = m.size_atom(), m.size_water()
    aa, aw, ww = g["aa"], g["aw"], g["ww_h"]
    # every ordered atom pair and every self term once (factor 2 on i<j, diagonal in bin 0)
    assert aa[1:, 1:].sum() == na * na and aw[1:].sum() == na * nw and ww.sum() == nw * nw
    if kind == 2:
        nx = len(m.exv)
        assert aa[1:, 0].sum() == na * nx and aa[0, 0].sum() == nx * nx and aw[0].sum() == nw * nx
    np.testing.assert_array_equal(g["q"], w.q)
    I, _ = O.debye_ff(kind, _ffhist(g), g["q"])
    np.testing.assert_allclose(I, g["Iq"], rtol=1e-12)


def test_batch_fixture():
    g = load_golden("fullsize_cfg3")
    w = synth.cfg3()
    assert len(w.molecules) == 256
    sizes = [w.molecules[int(i)].size_atom() for i in g["indices"]]
    assert sizes == sorted(sizes, reverse=True) and sizes[0] > 40000 and sizes[-1] < 1000
    for k, i in enumerate(g["indices"]):
        m = w.molecules[int(i)]
        assert input_digest(m) == str(g[f"digest{k}"])
        na, nw = m.size_atom(), m.size_water()
        assert g[f"aa{k}"][1:, 1:].sum() == na * na and g[f"ww_h{k}"].sum() == nw * nw
        I, _ = O.debye_ff(0, _ffhist(g, str(k)), g["q" + str(k)])
        np.testing.assert_allclose(I, g[f"Iq{k}"], rtol=1e-12)
