"""fitter::SmartFitter on the device (source/core/fitter/SmartFitter.cpp, include/core/fitter/SmartFitter.h).

The reference fits the enabled free parameters of a composite histogram to a measured profile with a
minimiser; a build without dlib uses mini::Golden, which fits one parameter.  Here the whole search
runs in one kernel on the unit profiles of one FP64 transform (ausaxs_gpu_fit).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import ctypes as C
import numpy as np

from . import _capi
from .hist import _Composite

# SmartFitter's parameter names (constants::fit::Parameters, include/core/constants/ConstantsFitParameters.h)
PARAMETERS = _capi.FIT_PARAMETERS


@dataclass
class FitResult:
    """The reference's FitResult for one fitted parameter plus the inner linear fit (a, b)."""

    parameter: str
    value: float
    a: float
    b: float
    a_err: float
    b_err: float
    chi2: float
    evaluations: int
    dof: int
    I_fit: np.ndarray

    def get_parameter_values(self):
        """[a, b, value], in the reference's order (the linear fit's parameters are added in front)."""
        return [self.a, self.b, self.value]


class SmartFitter:
    """SmartFitter(data, model): data = (q, I, sigma); model = a composite histogram returned by one of
    the managers in ausaxs_b200.hist.  Its current free parameters (apply_*_scaling_factor,
    apply_*_debye_waller_factor) are the values of the parameters that are not fitted."""

    def __init__(self, data: Tuple[Sequence[float], Sequence[float], Sequence[float]], model: _Composite):
        q, I, sigma = (np.ascontiguousarray(x, np.float64) for x in data)
        if not (len(q) == len(I) == len(sigma)):
            raise ValueError("q, I and sigma must have the same length")
        self.q, self.I, self.sigma = q, I, sigma
        self.model = model

    def fit(self, parameter: str = "cw", limits: Optional[Tuple[float, float]] = None,
            tolerance: float = 1e-4) -> FitResult:
        """Golden search of `parameter` within `limits` (default: the reference's limits for it)."""
        m = self.model
        f = m.free
        base = _capi.DebyeParams(f["cw"], f["cx"], f["crho"], f["dw_atomic"], f["dw_exv"], m.grid_width, 1, 0.0)
        lo, hi = limits if limits is not None else (0.0, 0.0)
        opt = _capi.FitOptions(PARAMETERS[parameter], lo, hi, tolerance)
        out = _capi.FitResult()
        I_fit = np.zeros(len(self.q))
        r = m._result()
        _capi.check(_capi.load().ausaxs_gpu_fit(m._ctx.h, C.byref(m._cfg), C.byref(r), _capi.dptr(self.q),
                                                _capi.dptr(self.I), _capi.dptr(self.sigma), len(self.q), C.byref(base),
                                                C.byref(opt), C.byref(out), _capi.dptr(I_fit)))
        return FitResult(parameter, out.value, out.a, out.b, out.a_err, out.b_err, out.chi2, out.evaluations,
                         len(self.q) - 3, I_fit)
