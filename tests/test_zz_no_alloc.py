"""The allocation-free Simple histogram (ausaxs_gpu_histogram_mt_noalloc) against ausaxs_gpu_histogram.

Some callers cannot allocate device memory while they run (memory-pool-managed or real-time code,
applications that forbid cudaMalloc after start-up because it can synchronise the device).  This
entry point serves them: device inputs, device outputs, and its temporaries in one file-scope device
array.  The test calls it twice in a row through the C ABI -- the second call must not see the
first call's leftovers in the shared array -- and compares both with the allocating entry point and
with the oracle, with weighted bins (distance sums per bin) and without.  This file is collected
last so that a failure here cannot hide other failures.
"""
import ctypes as C

import numpy as np
import pytest

from ausaxs_b200 import _capi, hist
from oracle import py as O

pytestmark = pytest.mark.gpu

W_RTOL = 1e-7  # weighted counts (fixed-point weight products), as tests/test_gpu_parity.py


def d_atol(bin_width):
    return bin_width * 2.0 ** -15


def _molecule(seed, na, nw):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(0, 10, (na, 3))
    w = rng.uniform(-0.5, 9.0, na)
    wat = rng.normal(0, 12, (nw, 3))
    ww = np.full(nw, 9.0)
    return hist.Molecule(atoms=xyz, weights=w, waters=wat, water_weights=ww)


def _noalloc(m, bin_width, bin_count, stream, weighted=1):
    import torch

    L = _capi.load()
    L.ausaxs_gpu_histogram_mt_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_double,
                                                  C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p]
    a, w = m.compact_w()
    da = torch.from_numpy(a).cuda()
    dw = torch.from_numpy(w).cuda()
    out = torch.full((5 * bin_count,), -1.0, dtype=torch.float64, device="cuda")
    mb = torch.zeros(1, dtype=torch.int32, device="cuda")
    of = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()  # inputs were written on the default stream
    rc = L.ausaxs_gpu_histogram_mt_noalloc(da.data_ptr(), len(a), dw.data_ptr(), len(w), bin_width, bin_count,
                                           int(weighted),
                                           out.data_ptr(), mb.data_ptr(), of.data_ptr(), stream.cuda_stream)
    _capi.check(rc)
    stream.synchronize()
    m_bin = int(mb.item())
    rows = out.cpu().numpy().reshape(5, bin_count)
    return m_bin, rows, int(of.item())


@pytest.mark.parametrize("weighted", [1, 0])
def test_noalloc_matches_allocating_entry_point_twice(weighted):
    import torch

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ctx = _capi.default_context(0)
    for seed, (na, nw, bw, nbins) in enumerate([(2500, 500, 0.25, 8000), (1300, 90, 0.1, 4000)]):
        m = _molecule(seed, na, nw)
        ref = hist.HistogramManagerMT(m, bool(weighted), bw, nbins, ctx).calculate_all()
        a, w = m.compact_w()
        orc = O.hist_simple(a, w, bw, nbins, weighted=bool(weighted))
        assert orc.overflow == 0 and len(orc.tot) == ref.max_bin
        for call in range(2):
            mb, rows, overflow = _noalloc(m, bw, nbins, stream, weighted)
            assert overflow == 0
            assert mb == ref.max_bin, (call, mb, ref.max_bin)
            aa, aw, ww, tot, d = (r[:mb] for r in rows)
            scale = np.abs(ref.get_aa_counts()).max()
            for got, want_gpu, want_oracle in ((aa, ref.get_aa_counts(), orc.aa), (aw, ref.get_aw_counts(), orc.aw),
                                               (ww, ref.get_ww_counts(), orc.ww), (tot, ref.get_counts(), orc.tot)):
                np.testing.assert_allclose(got, want_gpu, rtol=W_RTOL, atol=1e-9 * scale)
                np.testing.assert_allclose(got, want_oracle, rtol=W_RTOL, atol=1e-9 * scale)
            np.testing.assert_allclose(d, ref.get_d_axis(), rtol=0, atol=d_atol(bw))
            np.testing.assert_allclose(d, orc.d_axis, rtol=0, atol=d_atol(bw))
            assert not rows[:, mb:].any(), "bins beyond max_bin must be zero"


def test_noalloc_rejects_too_many_bins():
    import torch

    m = _molecule(9, 50, 5)
    with pytest.raises(_capi.AusaxsError) as e:
        _noalloc(m, 0.25, 9000, torch.cuda.Stream())
    assert e.value.code == _capi.ERR_CAPACITY
