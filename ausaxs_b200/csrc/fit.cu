// fitter::SmartFitter::fit() (source/core/fitter/SmartFitter.cpp:147-176) on the device, with the
// minimiser of a build without dlib: mini::Golden over one parameter (source/core/mini/Golden.cpp:26-74).
//
// The reference re-evaluates debye_transform() for every trial value; its sinc sums are cached, so a
// trial only recombines them with the parameter-dependent factors
// (CompositeDistanceHistogramFFAvgBase.cpp:377-397).  Here the recombination is taken one step
// further: every free parameter enters I(q) through per-q scalars on the six partial profiles
// evaluated at cw = cx = crho = 1 without Debye-Waller factors (the "unit profiles", one FP64
// transform):
//     aa = ba^2 P_aa            ax = crho c ba bx P_ax      xx = (c crho)^2 bx^2 P_xx
//     aw = cw ba P_aw           wx = crho c cw bx P_wx      ww = cw^2 P_ww
//     I  = aa - ax + aw + xx - wx + ww
// with ba = exp(-q^2 dw_atomic^2 / 2), bx = exp(-q^2 dw_exv^2 / 2), and c = cx (FFAvg, FFGrid) or
// c = exv_factor(q) = cx^3 exp(-(1.62^2/4)(cx^2 - 1) q^2) (FFExplicit, which is 1 at cx = 1); the
// Simple histogram has I = P_aa + cw P_aw + cw^2 P_ww.  Each trial is then the linear fit
// data ~ a I + b with weights 1/sigma^2 and chi2 = sum ((data - (a I + b)) / sigma)^2
// (fitter::detail::LinearLeastSquares, LinearLeastSquares.cpp:26-78).
//
// One CTA runs the whole search: every thread executes the same Golden control flow on the
// block-wide chi2 values, so no state is broadcast.  The sums that do not depend on the trial
// (S = sum w, Sy = sum w y, Syy = sum w y^2, w = 1/sigma^2) are formed once; a trial needs Sx, Sxx and
// Sxy only, one block reduction, and its chi2 follows from the sums,
//     chi2 = Syy - 2 a Sxy - 2 b Sy + a^2 Sxx + 2 a b Sx + b^2 S,
// which at the fitted value is recomputed as the reference forms it (explicit residuals).  The
// interval arithmetic is written with explicit round-to-nearest operations (no contraction), as the
// host evaluates it.
#include <cmath>

#include "common.cuh"
#include "fit.cuh"

namespace ausaxs_b200 {
namespace {

constexpr int kFitThreads = 256;
constexpr int kFitWarps = kFitThreads / 32;

// block-wide sum of N values; every thread gets the totals
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double (*s)[kFitWarps]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i)
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
    if (lane == 0)
#pragma unroll
        for (int i = 0; i < N; ++i) s[i][warp] = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < N; ++i) {
        double t = 0;
        for (int w = 0; w < kFitWarps; ++w) t += s[i][w];  // same order in every thread
        v[i] = t;
    }
    __syncthreads();
}

__device__ double model_intensity(const FitArgs& F, const double (&p)[5], int k) {
    const double* P = F.P;
    const int n = F.nq;
    const double cw = p[0];
    if (F.model == kFitSimple) return P[k] + cw * P[2 * n + k] + cw * cw * P[5 * n + k];
    const double q = F.q[k];
    const double cx = p[1], crho = p[2];
    const bool dw = p[3] != 0 || p[4] != 0;
    const double ba = dw ? exp(-q * q * p[3] * p[3] * 0.5) : 1.0;
    const double bx = dw ? exp(-q * q * p[4] * p[4] * 0.5) : 1.0;
    double c = cx;
    if (F.model == kFitExplicitExv) {
        const double rm2 = 1.62 * 1.62 / 4;  // exv_factor (CompositeDistanceHistogramFFExplicitBase.cpp:54-57)
        c = cx * cx * cx * exp(-rm2 * (cx * cx - 1) * q * q);
    }
    double I = 0;
    I += ba * ba * P[k];
    I -= crho * c * ba * bx * P[n + k];
    I += cw * ba * P[2 * n + k];
    I += (c * crho) * (c * crho) * bx * bx * P[3 * n + k];
    I -= crho * c * cw * bx * P[4 * n + k];
    I += cw * cw * P[5 * n + k];
    return I;
}

__global__ void __launch_bounds__(kFitThreads) fit_kernel(FitArgs F) {
    __shared__ double s_red[3][kFitWarps];
    const int n = F.nq;
    // trial-independent sums; w = 1/sigma^2 kept in the scratch array W
    double fixed[3] = {0, 0, 0};  // S, Sy, Syy
    for (int k = threadIdx.x; k < n; k += kFitThreads) {
        const double is = 1. / F.sigma[k];
        const double w = is * is;
        F.W[k] = w;
        fixed[0] += w;
        fixed[1] += F.y[k] * w;
        fixed[2] += F.y[k] * F.y[k] * w;
    }
    block_sum<3>(fixed, s_red);
    const double S = fixed[0], Sy = fixed[1], Syy = fixed[2];
    double fit_a = 0, fit_b = 0, Sx = 0, Sxx = 0, delta = 1;
    // chi2 of one trial value from the sums, identical in every thread
    auto evaluate = [&](double v) -> double {
        double p[5] = {F.base[0], F.base[1], F.base[2], F.base[3], F.base[4]};
        p[F.param] = v;
        double t[3] = {0, 0, 0};  // Sx, Sxx, Sxy
        for (int k = threadIdx.x; k < n; k += kFitThreads) {
            const double x = model_intensity(F, p, k);
            const double w = F.W[k];
            t[0] += x * w;
            t[1] += x * x * w;
            t[2] += x * F.y[k] * w;
        }
        block_sum<3>(t, s_red);
        Sx = t[0];
        Sxx = t[1];
        delta = S * Sxx - Sx * Sx;
        fit_a = (S * t[2] - Sx * Sy) / delta;
        fit_b = (Sxx * Sy - Sx * t[2]) / delta;
        return Syy - 2 * fit_a * t[2] - 2 * fit_b * Sy + fit_a * fit_a * Sxx + 2 * fit_a * fit_b * Sx +
               fit_b * fit_b * S;
    };
    // the final evaluation as the reference forms it: the sums, then the explicit residuals
    auto evaluate_residuals = [&](double v) -> double {
        evaluate(v);
        double p[5] = {F.base[0], F.base[1], F.base[2], F.base[3], F.base[4]};
        p[F.param] = v;
        double c2[1] = {0};
        for (int k = threadIdx.x; k < n; k += kFitThreads) {
            const double x = model_intensity(F, p, k);
            F.Iw[k] = x;
            const double r = (F.y[k] - (fit_a * x + fit_b)) * (1. / F.sigma[k]);
            c2[0] += r * r;
        }
        block_sum<1>(c2, s_red);
        return c2[0];
    };

    // Golden::search
    double a = F.lo, b = F.hi;
    const double temp = __dadd_rn(a, b);
    a = fmin(a, b);
    b = __dsub_rn(temp, a);
    double diff = __dsub_rn(b, a), ilo = a, ihi = b;
    int evaluations = 0;
    if (F.steps >= 0) {
        double c = __dadd_rn(a, __dmul_rn(F.invphi2, diff)), d = __dadd_rn(a, __dmul_rn(F.invphi, diff));
        double fc = evaluate(c), fd = evaluate(d);
        evaluations = 2;
        for (int k = 0; k < F.steps - 1; ++k) {
            if (fc < fd) {
                b = d;
                d = c;
                fd = fc;
                diff = __dmul_rn(F.invphi, diff);
                c = __dadd_rn(a, __dmul_rn(F.invphi2, diff));
                fc = evaluate(c);
            } else {
                a = c;
                c = d;
                fc = fd;
                diff = __dmul_rn(F.invphi, diff);
                d = __dadd_rn(a, __dmul_rn(F.invphi, diff));
                fd = evaluate(d);
            }
            ++evaluations;
        }
        if (fc < fd) ilo = a, ihi = d;
        else ilo = c, ihi = b;
    }
    // Golden::minimize_override: the centre of the final interval (Limit::center = min + span / 2)
    const double value = __dadd_rn(ilo, __dsub_rn(ihi, ilo) / 2);
    const double chi2 = evaluate_residuals(value);
    if (F.I_fit)
        for (int k = threadIdx.x; k < n; k += kFitThreads) F.I_fit[k] = fit_a * F.Iw[k] + fit_b;
    if (threadIdx.x == 0) {
        F.out[0] = value;
        F.out[1] = fit_a;
        F.out[2] = fit_b;
        F.out[3] = chi2;
        F.out[4] = evaluations;  // as the reference counts them: without the evaluation at value
        F.out[5] = sqrt(S / delta);
        F.out[6] = sqrt(Sxx / delta);
    }
}

}  // namespace

void fit_launch(const FitArgs& F, cudaStream_t s) { fit_kernel<<<1, kFitThreads, 0, s>>>(F); }

}  // namespace ausaxs_b200
