// Weighted linear least squares + chi-square (see lsq.cu).
#pragma once
#include <cuda_runtime.h>

namespace ausaxs_b200 {
// out[5] = {a, b, sigma_a, sigma_b, chi2} for model ~ a * data + b with weights 1/err^2 (device pointers).
void lsq_launch(const double* data, const double* model, const double* err, int n, double* out, cudaStream_t s);
}  // namespace ausaxs_b200
