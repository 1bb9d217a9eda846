// Measurement kernels for the roofline of the pair kernel (no counterpart in the reference).
//
// The pair kernel's work per pair is a handful of FP32 operations plus two 32-bit shared-memory
// atomics (count, fixed-point distance offset).  Its roofline takes the lower of the FP32 bound and
// the shared-atomic bound; the second is measured here: every resident thread adds 1 to a shared
// 32-bit word with atomicAdd, the lanes of a warp on distinct banks (lane + 32 * k, k drawn per
// thread and iteration from a small generator), so the rate is the shared-atomic throughput without
// bank conflicts.  A second mode draws the bin uniformly at random over the array (conflicts as they
// happen), the pair kernel's own situation with uncorrelated distances.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/ausaxs_b200_diag.h"

namespace ausaxs_b200 {
void set_last_error(const char* msg);  // capi.cu

namespace {

constexpr int kDiagBins = 4096;  // u32 words per CTA (16 KB), a typical on-chip histogram size
constexpr int kDiagThreads = 512;
constexpr int kDiagUnroll = 8;

// W64: 64-bit atomicAdd on an array of the same byte size (kDiagBins / 2 words)
template <bool W64>
__global__ void __launch_bounds__(kDiagThreads) smem_atomic_kernel(int iters, int conflict_free, unsigned* sink) {
    using T = typename std::conditional<W64, unsigned long long, unsigned>::type;
    constexpr int kWords = W64 ? kDiagBins / 2 : kDiagBins;
    __shared__ T h[kWords];
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) h[k] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31u;
    unsigned x = 0x9E3779B9u * (blockIdx.x * blockDim.x + threadIdx.x + 1u);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < kDiagUnroll; ++u) {
            x = x * 1664525u + 1013904223u;  // LCG (Numerical Recipes constants)
            const unsigned r = x >> 20;      // 12 random bits
            const unsigned b = conflict_free ? (lane | ((r & (kWords / 32 - 1)) << 5)) : (r & (kWords - 1));
            atomicAdd(&h[b], static_cast<T>(1));
        }
    }
    __syncthreads();
    T s = 0;
    for (int k = threadIdx.x; k < kWords; k += blockDim.x) s += h[k];
    if (s == static_cast<T>(0xFFFFFFFFu)) sink[0] = static_cast<unsigned>(s);  // keeps the atomics alive; never true in practice
}

int fail(int code, const char* msg) {
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace ausaxs_b200

using namespace ausaxs_b200;

extern "C" int ausaxs_gpu_smem_atomic_rate(int32_t device, int32_t conflict_free, double* atomics_per_s, double* ms) {
    if (!atomics_per_s) return fail(AUSAXS_ERR_ARGUMENT, "null argument");
    cudaGetLastError();
    if (cudaSetDevice(device) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, "no such device");
    const bool w64 = (conflict_free & 2) != 0;
    const int mode = conflict_free & 1;
    auto kernel = w64 ? smem_atomic_kernel<true> : smem_atomic_kernel<false>;
    int sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return fail(AUSAXS_ERR_CUDA, "cannot query the multiprocessor count");
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kDiagThreads, 0) != cudaSuccess || per_sm <= 0)
        return fail(AUSAXS_ERR_CUDA, "cannot query the occupancy");
    unsigned* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = AUSAXS_OK;
    const int grid = sms * per_sm;
    const int iters = 4096;
    float t = 0;
    if (cudaMalloc(&sink, sizeof(unsigned)) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = fail(AUSAXS_ERR_CUDA, "cannot allocate the measurement's resources");
    } else {
        kernel<<<grid, kDiagThreads, 0, s>>>(iters / 8, mode, sink);  // warm-up
        cudaEventRecord(e0, s);
        kernel<<<grid, kDiagThreads, 0, s>>>(iters, mode, sink);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess || t <= 0)
            rc = fail(AUSAXS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
    if (rc == AUSAXS_OK) {
        *atomics_per_s = (double)grid * kDiagThreads * (double)iters * kDiagUnroll / (t * 1e-3);
        if (ms) *ms = t;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (sink) cudaFree(sink);
    return rc;
}
