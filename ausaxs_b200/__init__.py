"""B200-native (sm_100a) implementation of AUSAXS's Debye hot path.

The weighted-bin pair-distance histograms and the form-factor-weighted Debye transform run as
hand-written CUDA kernels behind a C ABI (include/ausaxs_b200.h); this package holds the kernels
(``csrc/``), their build (``build``), the ctypes binding (``_capi``) and a host-side mirror of the
reference's histogram-manager interfaces (``hist``).
"""
from .hist import (CompositeDistanceHistogram, CompositeDistanceHistogramFFAvg, CompositeDistanceHistogramFFExplicit,
                   CompositeDistanceHistogramFFGrid, HistogramManagerMT, HistogramManagerMTFFAvg,
                   HistogramManagerMTFFExplicit, HistogramManagerMTFFGrid, Molecule, default_q_axis, profile)

__all__ = [
    "Molecule", "HistogramManagerMT", "HistogramManagerMTFFAvg", "HistogramManagerMTFFExplicit",
    "HistogramManagerMTFFGrid", "CompositeDistanceHistogram", "CompositeDistanceHistogramFFAvg",
    "CompositeDistanceHistogramFFExplicit", "CompositeDistanceHistogramFFGrid", "default_q_axis", "profile",
]
