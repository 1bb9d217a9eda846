"""The reference's own code over the device path, compiled from its sources (oracle/Makefile target
`adapter`): HistogramManagerMT, PartialHistogramManagerMT and SymmetryManagerMT issuing their pair work
to the device SimpleCalculator (oracle/adapter/shim), and the device HistogramManagerMTFFAvg
(oracle/adapter/gpu_adapter.h) feeding the reference's CompositeDistanceHistogramFFAvg and its
debye_transform().  The same workload (tests/adapter_run.py: symmetric molecules with a c3 and a
tetrahedral symmetry, a three-body molecule, three steps of rigid moves, an FFAvg molecule) runs once
on the reference's CPU classes and once on the adapter build, each in a process of its own.

Bar: FF pair counts exact; weighted counts within 1e-6 relative (the device quantises each weight
product to 2^-30 of the largest); distance axes within the fixed-point offset resolution plus the
reference's own float rounding of the distance sums; I(q) from the reference's transform within 1e-6."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BW = 0.25


def _run(tmp_path, lib):
    out = str(tmp_path / f"{lib}.npz")
    env = dict(os.environ, AUSAXS_REF_LIB=lib)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "adapter_run.py"), out], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    with np.load(out) as z:
        return {k: z[k] for k in z.files}


def _d_bound(n):
    return BW * 2.0 ** -15 + (np.arange(n) + 1) * BW * 2.0 ** -24 + 1e-9


def test_reference_managers_over_the_device_calculator(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libausaxs_ref_gpu.so")):
        pytest.fail("the adapter build is missing: make -C oracle adapter")
    cpu = _run(tmp_path, "libausaxs_ref.so")
    gpu = _run(tmp_path, "libausaxs_ref_gpu.so")
    assert int(cpu["adapter"]) == 0 and int(gpu["adapter"]) == 1
    keys = [k for k in cpu if k.endswith("_tot") or k in ("mt_aa", "mt_aw", "mt_ww")]
    for k in keys:
        a, b = gpu[k], cpu[k]
        assert a.shape == b.shape, (k, a.shape, b.shape)
        if k.startswith("ff_"):
            np.testing.assert_array_equal(a, b, err_msg=k)
        else:
            np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-9 * np.abs(b).max(), err_msg=k)
    for k in [k for k in cpu if k.endswith("_d")]:
        a, b = gpu[k], cpu[k]
        assert np.all(np.abs(a - b) <= _d_bound(len(b))), k
    for k in ("ff_aa", "ff_aw", "ff_ww"):
        np.testing.assert_array_equal(gpu[k], cpu[k], err_msg=k)
    for k in [k for k in cpu if k.endswith("_I")]:
        np.testing.assert_allclose(gpu[k], cpu[k], rtol=1e-6, atol=0, err_msg=k)
    np.testing.assert_allclose(gpu["ff_prof"], cpu["ff_prof"], rtol=1e-6, atol=1e-9 * np.abs(cpu["ff_prof"]).max())
