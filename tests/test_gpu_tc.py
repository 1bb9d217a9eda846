"""Split-BF16 tensor-core Debye contraction (precision 0) against the FP64 path and the oracle.

Bar: with precision 0 every q either keeps its tensor-core value, when the rigorous error bound the
kernel forms is within the tolerance, or is re-evaluated in FP64; so I(q) is within the tolerance
(1e-4 relative, the path's stated I(q) bar) of the FP64 result everywhere.  The bound itself is
checked: with an infinite tolerance (tensor-core values only) the actual deviation from FP64 never
exceeds it.
"""
import numpy as np
import pytest

from ausaxs_b200 import hist, synth
from oracle import py as O
from tests.helpers import golden_cases, load_golden
from tests.test_gpu_parity import manager_for

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _pair(h, q, ctx, tolerance):
    h.precision, h.tolerance = 1, 1e-5
    _, I64 = h.debye_transform(q)
    p64 = h.profiles(q)
    h.precision, h.tolerance = 0, tolerance
    _, Itc = h.debye_transform(q)
    return I64, p64, Itc


def _cases(ctx):
    out = []
    for name in golden_cases():
        g = load_golden(name)
        h = manager_for(g, ctx).calculate_all()
        cw, cx, crho, dwa, dwx = g["params"]
        h.apply_water_scaling_factor(cw)
        if str(g["manager"]) != "mt":
            h.apply_excluded_volume_scaling_factor(cx)
            h.apply_solvent_density_scaling_factor(crho)
            h.apply_atomic_debye_waller_factor(dwa)
            h.apply_exv_debye_waller_factor(dwx)
        out.append((name, h, np.asarray(g["q"])))
    w = synth.cfg0()
    out.append(("cfg0", hist.HistogramManagerMTFFAvg(w.molecules[0], True, 0.25, 8000, ctx).calculate_all(), w.q))
    rng = np.random.default_rng(3)
    xyz = rng.normal(0, 14, (3000, 3))
    ff = rng.choice([3, 7, 11, 12], 3000).astype(np.int32)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=rng.normal(0, 16, (600, 3)),
                      exv=np.round(rng.uniform(-14, 14, (4000, 3))), volume=1.0)
    out.append(("ffgrid", hist.HistogramManagerMTFFGrid(m, 0.1, 8000, ctx).calculate_all(),
                np.linspace(0.002, 1.0, 700)))
    return out


def test_tc_bound_covers_actual_error(gpu_ctx):
    worst = 0.0
    for name, h, q in _cases(gpu_ctx):
        I64, _, Itc = _pair(h, q, gpu_ctx, 1e30)
        assert gpu_ctx.fp64_columns() == 0, name
        est = gpu_ctx.tc_error_estimate(len(q))
        assert np.all(np.isfinite(est) | (Itc == 0)), name
        dev = np.abs(Itc - I64) / np.maximum(np.abs(Itc), 1e-300)
        ok = dev <= est
        assert ok.all(), (name, np.flatnonzero(~ok)[:5], dev[~ok][:5], est[~ok][:5])
        worst = max(worst, float(np.max(dev / np.maximum(est, 1e-300))))
    print(f"largest actual/bound ratio {worst:.3g}")


def test_tc_within_tolerance_of_fp64(gpu_ctx):
    for name, h, q in _cases(gpu_ctx):
        I64, _, Itc = _pair(h, q, gpu_ctx, TOL)
        np.testing.assert_allclose(Itc, I64, rtol=TOL, atol=0, err_msg=name)
        n64 = gpu_ctx.fp64_columns()
        assert 0 <= n64 <= len(q)
        print(f"{name}: {n64}/{len(q)} q in FP64")


def test_tc_profile_vs_oracle_cfg0(gpu_ctx):
    w = synth.cfg0()
    m = w.molecules[0]
    mgr = hist.HistogramManagerMTFFAvg(m, True, 0.25, 8000, gpu_ctx)
    I = hist.profile(mgr, w.q, precision=0, tolerance=TOL)
    A, W, _ = m.compact_ff()
    o = O.hist_ff(0, A, W, None, 0.25, 8000, m.volume * 0.334 / m.size_atom())
    Io, _ = O.debye_ff(0, o, w.q)
    np.testing.assert_allclose(I, Io, rtol=TOL)


def test_tc_large_counts_and_many_bins(gpu_ctx):
    # 20,000 atoms at 0.1 A bins: counts up to ~1e5 per bin and ~1,500 bins in use
    rng = np.random.default_rng(8)
    xyz = rng.normal(0, 25, (20000, 3))
    ff = rng.choice([3, 7, 11], 20000).astype(np.int32)
    m = hist.Molecule(atoms=xyz, ff_types=ff, waters=rng.normal(0, 28, (2000, 3)), volume=20000 * 18.0)
    h = hist.HistogramManagerMTFFAvg(m, True, 0.1, 8000, gpu_ctx).calculate_all()
    q = np.linspace(1e-4, 1.0, 1000)
    I64, _, Itc = _pair(h, q, gpu_ctx, TOL)
    np.testing.assert_allclose(Itc, I64, rtol=TOL, atol=0)
    I64, _, Itc = _pair(h, q, gpu_ctx, 1e30)
    est = gpu_ctx.tc_error_estimate(len(q))
    assert np.all(np.abs(Itc - I64) <= est * np.abs(Itc))


def test_automatic_precision_picks_by_size(gpu_ctx):
    """precision 2: FP64 for a small transform (every q counted as FP64), tensor cores for a large one."""
    g = load_golden("random0_ffavg")
    h = manager_for(g, gpu_ctx).calculate_all()
    h.precision, h.tolerance = 2, TOL
    q = np.asarray(g["q"])
    _, I2 = h.debye_transform(q)
    assert gpu_ctx.fp64_columns() == len(q) and not np.isfinite(gpu_ctx.tc_error_estimate(len(q))).any()
    h.precision = 1
    _, I1 = h.debye_transform(q)
    np.testing.assert_array_equal(I2, I1)
    rng = np.random.default_rng(8)
    xyz = rng.normal(0, 25, (20000, 3))
    m = hist.Molecule(atoms=xyz, ff_types=rng.choice([3, 7, 11], 20000).astype(np.int32),
                      waters=rng.normal(0, 28, (2000, 3)), volume=20000 * 18.0)
    h = hist.HistogramManagerMTFFAvg(m, True, 0.1, 8000, gpu_ctx).calculate_all()
    h.precision, h.tolerance = 2, TOL
    q = np.linspace(1e-4, 1.0, 1000)
    _, I2 = h.debye_transform(q)
    # the contraction ran: its error bounds were formed (how many q it keeps depends on the bound)
    assert np.isfinite(gpu_ctx.tc_error_estimate(len(q))).any()
    h.precision = 1
    _, I1 = h.debye_transform(q)
    np.testing.assert_allclose(I2, I1, rtol=TOL)


def _exact_pair(h, q, ctx, tolerance):
    h.precision, h.tolerance = 1, 1e-5
    _, I64 = h.debye_transform(q)
    h.precision, h.tolerance = 3, tolerance
    _, Ix = h.debye_transform(q)
    return I64, Ix, ctx.fp64_columns(), ctx.tc_error_estimate(len(q))


@pytest.mark.parametrize("grid", [False, True])
def test_exact_tensor_core_transform(gpu_ctx, grid):
    """precision 3: int8 digit products (exact s32 sums) of the histogram rows and of shared Taylor
    tables.  The rigorous bound keeps (almost) every q on the tensor cores at the 1e-4 bar, the actual
    deviation from the FP64 transform stays below the bound, and far below the bar."""
    rng = np.random.default_rng(21 + grid)
    n = 6000
    xyz = rng.normal(0, 14, (n, 3))
    m = hist.Molecule(atoms=xyz, ff_types=rng.choice([3, 7, 11, 12], n).astype(np.int32),
                      waters=rng.normal(0, 17, (1200, 3)), volume=n * 18.0,
                      exv=np.round(rng.uniform(-15, 15, (3000, 3))) if grid else None)
    w = 0.1
    h = (hist.HistogramManagerMTFFGrid(m, w, 8000, gpu_ctx) if grid
         else hist.HistogramManagerMTFFAvg(m, True, w, 8000, gpu_ctx)).calculate_all()
    if grid:
        h.apply_excluded_volume_scaling_factor(1.07)
    q = np.linspace(0.005, 1.0, 1000)
    I64, Ix, n64, est = _exact_pair(h, q, gpu_ctx, TOL)
    rel = np.abs(Ix / I64 - 1)
    assert np.max(rel) <= TOL
    assert n64 <= 0.02 * len(q), n64
    kept = np.isfinite(est) & (est <= TOL)
    assert np.all(rel[kept] <= est[kept])  # the bound holds
    # the digits and the integer sums leave about 1e-11; the Taylor truncation, held below 2^-32 of
    # sum |H|, dominates at high q where I(q) is small against sum |H|
    assert np.median(rel) < 1e-6
    # repeated transforms on the same q grid reuse the tables and give the same bits
    _, Ix2, _, _ = _exact_pair(h, q, gpu_ctx, TOL)
    np.testing.assert_array_equal(Ix2, Ix)
    # a new q grid at the same address (the context's staging buffer) rebuilds them
    q2 = np.linspace(0.01, 0.9, 1000)
    I64b, Ixb, _, _ = _exact_pair(h, q2, gpu_ctx, TOL)
    assert np.max(np.abs(Ixb / I64b - 1)) <= TOL


def test_exact_transform_on_golden_cases(gpu_ctx):
    """precision 3 against the FP64 transform on every golden case (their parameters applied)."""
    for name, h, q in _cases(gpu_ctx):
        h.precision, h.tolerance = 1, 1e-5
        _, I64 = h.debye_transform(q)
        h.precision, h.tolerance = 3, TOL
        _, I = h.debye_transform(q)
        np.testing.assert_allclose(I, I64, rtol=TOL, err_msg=name)
