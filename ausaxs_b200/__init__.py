"""B200-native (sm_100a) implementation of AUSAXS's Debye hot path.

The weighted-bin pair-distance histograms and the form-factor-weighted Debye transform run as
hand-written CUDA kernels behind a C ABI (include/ausaxs_b200.h); this package holds the kernels
(``csrc/``), their build (``build``), the ctypes binding (``_capi``), a host-side mirror of the
reference's histogram-manager interfaces (``hist``) and of its fitter (``fitter``).
"""
from .hist import (CompositeDistanceHistogram, CompositeDistanceHistogramFFAvg, CompositeDistanceHistogramFFExplicit,
                   CompositeDistanceHistogramFFGrid, HistogramManagerMT, HistogramManagerMTFFAvg,
                   HistogramManagerMTFFExplicit, HistogramManagerMTFFGrid, Molecule, default_q_axis, profile)

from ._capi import Calculator
from .fitter import FitResult, SmartFitter

__all__ = [
    "Calculator", "SmartFitter", "FitResult",
    "Molecule", "HistogramManagerMT", "HistogramManagerMTFFAvg", "HistogramManagerMTFFExplicit",
    "HistogramManagerMTFFGrid", "CompositeDistanceHistogram", "CompositeDistanceHistogramFFAvg",
    "CompositeDistanceHistogramFFExplicit", "CompositeDistanceHistogramFFGrid", "default_q_axis", "profile",
]
