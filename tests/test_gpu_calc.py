"""The device SimpleCalculator (scaled self/cross jobs with merge ids) against the reference's own
calculator runs and the oracle.

Bar: counts exact; weighted values within the fixed-point resolution of the weight products (each
pair's w_i w_j is quantised to 2^-k with max|w|^2 2^k <= 2^30: |error| <= 2^-31 max|w|^2 per pair);
distance sums within count * c * 2^-15 (the in-bin offset of a pair is quantised to c * 2^-15) plus the
reference's own float rounding of factor * distance."""
import numpy as np
import pytest

from ausaxs_b200 import _capi
from oracle import py as O
from tests.helpers import calc_cases, calc_inputs, load_golden

pytestmark = pytest.mark.gpu


def run_gpu(ctx, sets, jobs, bin_width):
    calc = _capi.Calculator(ctx, bin_width, 8000)
    idx = []
    for a, b, sc, m in jobs:
        if b is None:
            idx.append(calc.enqueue_calculate_self(sets[a], sc, m))
        else:
            idx.append(calc.enqueue_calculate_cross(sets[a], sets[b], sc, m))
    out = calc.run()
    calc.close()
    return out, idx


def within(x, ref, bound, what):
    bad = np.abs(x - ref) > bound
    assert not np.any(bad), f"{what}: {np.count_nonzero(bad)} bins, worst excess {np.max(np.abs(x - ref) - bound):.3g}"


def check_result(res, ref, sets, bin_width, nbins):
    v, c, d = (x[:nbins] for x in res)
    rv, rc, rd = ref
    np.testing.assert_array_equal(c, rc)
    # the weight scale is the largest 2^k with max|w|^2 2^k <= 2^30, so a product's quantisation error is
    # at most max|w|^2 2^-30, and a bin's value carries count (= 2 scaling pairs) of them
    wmax2 = max(float(np.max(np.abs(s[:, 3]))) ** 2 for s in sets)
    within(v, rv, (rc + 1) * wmax2 * 2.0 ** -30 + 1e-12 * np.abs(rv).max(), "value")
    # the device sums each pair's distance exactly; the reference adds N * distance rounded to float
    # (WeightedEntry.h:77-81), i.e. up to N d 2^-24 per pair with d < (bin + 1) * width
    d_bound = rc * bin_width * 2.0 ** -15 + rc * (np.arange(len(rc)) + 1) * bin_width * 2.0 ** -24 + 1e-9
    within(d, rd, d_bound, "distance sum")


@pytest.mark.parametrize("name", calc_cases())
def test_calculator_vs_reference(name, gpu_ctx):
    g = load_golden(name)
    sets, jobs = calc_inputs(g)
    bw = float(g["bin_width"])
    out, _ = run_gpu(gpu_ctx, sets, jobs, bw)
    keys = [tuple(int(x) for x in k) for k in g["keys"]]
    assert sorted((0, i) for i in out["self"]) + sorted((1, i) for i in out["cross"]) == keys
    n = g["results"].shape[2]
    for r, (cross, mid) in enumerate(keys):
        res = out["cross" if cross else "self"][mid]
        check_result(res, g["results"][r], sets, bw, n)
        assert not np.any(res[1][n:])


def test_result_indices_follow_the_reference(gpu_ctx):
    rng = np.random.default_rng(4)
    s = [np.column_stack([rng.normal(0, 5, (40, 3)), rng.uniform(1, 2, 40)]).astype(np.float32) for _ in range(3)]
    jobs = [(0, None, 1, 5), (1, None, 1, -1), (2, None, 2, 5), (0, 1, 1, -1), (1, 2, 1, 0), (0, 2, 3, 1), (2, 0, 1, 1)]
    out, idx = run_gpu(gpu_ctx, s, jobs, 0.25)
    # self: id 5 -> 0, -1 -> a new result with id 1; cross: -1 -> id 0, then 0 merges into it, 1 -> 1
    assert idx == [0, 1, 0, 0, 0, 1, 1]
    assert sorted(out["self"]) == [1, 5] and sorted(out["cross"]) == [0, 1]
    o = O.calculator(s, jobs, 0.25, 8000)
    for (cross, mid), ref in o.items():
        check_result(out["cross" if cross else "self"][mid], ref, s, 0.25, 8000)


def test_scaling_is_a_multiplicity(gpu_ctx):
    rng = np.random.default_rng(5)
    a = np.column_stack([rng.normal(0, 8, (700, 3)), rng.uniform(0.5, 6, 700)]).astype(np.float32)
    b = np.column_stack([rng.normal(3, 8, (300, 3)), rng.uniform(0.5, 6, 300)]).astype(np.float32)
    one, _ = run_gpu(gpu_ctx, [a, b], [(0, None, 1, 0), (0, 1, 1, 0)], 0.1)
    sev, _ = run_gpu(gpu_ctx, [a, b], [(0, None, 7, 0), (0, 1, 7, 0)], 0.1)
    for key in ("self", "cross"):
        v1, c1, d1 = one[key][0]
        v7, c7, d7 = sev[key][0]
        np.testing.assert_array_equal(c7[1:], 7 * c1[1:])
        np.testing.assert_allclose(v7[1:], 7 * v1[1:], rtol=1e-14)
        np.testing.assert_allclose(d7[1:], 7 * d1[1:], rtol=1e-14)


def test_calculator_errors(gpu_ctx):
    calc = _capi.Calculator(gpu_ctx, 0.25, 8000)
    p = np.zeros((3, 4), np.float32)
    with pytest.raises(_capi.AusaxsError):
        calc.enqueue_calculate_self(p, 0, 0)  # scaling must be positive
    calc.enqueue_calculate_self(p, 1, 0)
    out = calc.run()
    assert list(out["self"]) == [0] and out["cross"] == {}
    with pytest.raises(_capi.AusaxsError) as e:
        v = np.zeros(8000)
        _capi.check(_capi.load().ausaxs_gpu_calculator_result(calc.h, 1, 3, _capi.dptr(v), _capi.dptr(v), _capi.dptr(v)))
    assert e.value.code == _capi.ERR_NOT_FOUND
    calc.close()


def test_calculator_empty_sets_and_repeated_runs(gpu_ctx):
    rng = np.random.default_rng(6)
    a = np.column_stack([rng.normal(0, 4, (50, 3)), rng.uniform(1, 2, 50)]).astype(np.float32)
    empty = np.zeros((0, 4), np.float32)
    calc = _capi.Calculator(gpu_ctx, 0.25, 8000)
    assert calc.run() == {"self": {}, "cross": {}}  # nothing enqueued
    calc.enqueue_calculate_self(empty, 2, 0)
    calc.enqueue_calculate_cross(a, empty, 1, 0)
    out = calc.run()
    assert not np.any(out["self"][0][0]) and not np.any(out["cross"][0][0])
    for _ in range(2):  # the same jobs twice give the same results (run clears the jobs)
        calc.enqueue_calculate_self(a, 3, 7)
        r = calc.run()
        assert list(r["self"]) == [7]
    o = O.calculator([a], [(0, None, 3, 7)], 0.25, 8000)
    check_result(r["self"][7], o[(0, 7)], [a], 0.25, 8000)
    calc.close()
