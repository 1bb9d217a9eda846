// Device-side fit of one free parameter of a composite histogram against measured data: the
// reference's fitter::SmartFitter with the minimiser of a build without dlib (mini::Golden), in one
// kernel (see fit.cu).
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace ausaxs_b200 {

// How the free parameters enter I(q) given the unit profiles (the six partial profiles at cw = cx =
// crho = 1 without Debye-Waller factors).
enum FitModel : int32_t {
    kFitAverageExv = 0,  // FFAvg and FFGrid: cx scales the excluded volume directly
    kFitExplicitExv = 1, // FFExplicit: cx enters through exv_factor(q) = cx^3 exp(-(r^2/4)(cx^2 - 1) q^2)
    kFitSimple = 2       // Simple (weights): I = aa + cw aw + cw^2 ww
};

struct FitArgs {
    int32_t model;         // FitModel
    int32_t nq;
    const double* q;       // [nq]
    const double* P;       // [6][nq] unit profiles {aa, ax, aw, xx, wx, ww}
    const double* y;       // [nq] measured intensities
    const double* sigma;   // [nq] their errors
    double base[5];        // cw, cx, crho, dw_atomic, dw_exv (the free one is replaced by the trial value)
    int32_t param;         // index of the free parameter
    double lo, hi;         // search interval
    int32_t steps;         // Golden iterations n = ceil(log(tol / (hi - lo)) / log(1 / phi)); < 0: no search
    double invphi, invphi2;
    double* Iw;            // [nq] scratch: model intensities at the fitted value
    double* W;             // [nq] scratch: 1 / sigma^2
    double* out;           // [7]: value, a, b, chi2, evaluations, a_err, b_err
    double* I_fit;         // [nq] or null: a I_model + b at the fitted value
};

void fit_launch(const FitArgs& F, cudaStream_t s);

}  // namespace ausaxs_b200
