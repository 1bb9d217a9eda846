"""The C-ABI library: it builds for sm_100a, loads, and exports every symbol include/*.h declares.
CPU only: no kernel is launched here."""
import glob
import os
import re
import subprocess

import pytest

from ausaxs_b200 import _capi
from ausaxs_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"AUSAXS_API\s+[\w\s\*]+?\b(ausaxs_\w+)\s*\(", text))
    return names


def test_build_and_exports():
    path = build()
    assert os.path.exists(path)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (ausaxs_\w+)", out))
    decl = declared_symbols()
    assert decl, "no declarations found"
    assert decl <= exported, f"declared but not exported: {sorted(decl - exported)}"
    assert set(_capi.EXPORTED) == decl


def test_library_loads_and_binds():
    L = _capi.load()
    for name in _capi.EXPORTED:
        assert hasattr(L, name)


def test_no_device_reports_error_not_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_capi.AusaxsError) as e:
        _capi.Context(0)
    assert e.value.code in (_capi.ERR_ARGUMENT, _capi.ERR_CUDA)
