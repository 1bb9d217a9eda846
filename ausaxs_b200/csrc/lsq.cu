// Closed-form weighted linear least squares and chi-square on the device (the K6 stage).
//
// fitter::detail::LinearLeastSquares::fit_params_only / fit (source/core/fitter/detail/
// LinearLeastSquares.cpp:26-55): fit model ~ a * data + b with weights 1/err^2, then
// chi2 = sum ((model - (a data + b)) / err)^2.  LinearFitter passes the measured intensities as
// `data` and the model spliced onto the measured q as `model` (source/core/fitter/LinearFitter.cpp:14-21).
// One CTA: FP64 block reductions of S, Sx, Sy, Sxx, Sxy, then a second pass for chi2.
#include "lsq.cuh"

namespace ausaxs_b200 {
namespace {

constexpr int kLsqThreads = 256;

__device__ double block_sum(double v, double* s_red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kLsqThreads / 32; ++w) t += s_red[w];
    __syncthreads();
    if (threadIdx.x == 0) s_red[0] = t;
    __syncthreads();
    return s_red[0];
}

__global__ void __launch_bounds__(kLsqThreads) lsq_kernel(const double* data, const double* model, const double* err,
                                                          int n, double* out) {
    __shared__ double s_red[kLsqThreads / 32];
    double S = 0, Sx = 0, Sy = 0, Sxx = 0, Sxy = 0;
    for (int i = threadIdx.x; i < n; i += kLsqThreads) {
        double is = 1.0 / err[i];
        double w = is * is;
        S += w;
        Sx += data[i] * w;
        Sy += model[i] * w;
        Sxx += data[i] * data[i] * w;
        Sxy += data[i] * model[i] * w;
    }
    S = block_sum(S, s_red);
    Sx = block_sum(Sx, s_red);
    Sy = block_sum(Sy, s_red);
    Sxx = block_sum(Sxx, s_red);
    Sxy = block_sum(Sxy, s_red);
    const double delta = S * Sxx - Sx * Sx;
    const double a = (S * Sxy - Sx * Sy) / delta;
    const double b = (Sxx * Sy - Sx * Sxy) / delta;
    double c2 = 0;
    for (int i = threadIdx.x; i < n; i += kLsqThreads) {
        double r = (model[i] - (a * data[i] + b)) / err[i];
        c2 += r * r;
    }
    c2 = block_sum(c2, s_red);
    if (threadIdx.x == 0) {
        out[0] = a;
        out[1] = b;
        out[2] = sqrt(S / delta);    // FitResult sigma_a (LinearLeastSquares.cpp:50)
        out[3] = sqrt(Sxx / delta);  // sigma_b
        out[4] = c2;
    }
}

}  // namespace

void lsq_launch(const double* data, const double* model, const double* err, int n, double* out, cudaStream_t s) {
    lsq_kernel<<<1, kLsqThreads, 0, s>>>(data, model, err, n, out);
}

}  // namespace ausaxs_b200
