// Point-set preparation: bounding box, form-factor type census and dense-type conversion.
//
// Mirrors CompactCoordinatesFF::setup (include/core/hist/detail/CompactCoordinatesFF.h:21-32):
// every atom's form-factor type is validated (UNKNOWN and out-of-range types are an error) and
// remapped, here to a dense index over the types the structure actually contains, so that the
// on-chip histograms hold T*T rows instead of 15*15.
#include "prep.cuh"

namespace ausaxs_b200 {

namespace {

// float <-> order-preserving uint32 (for atomicMin/atomicMax on floats)
__device__ __forceinline__ unsigned int f2o(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void census_kernel(const float4* p, int n, int ff_typed, PrepStats* st) {
    __shared__ unsigned int s_lo[3], s_hi[3], s_mask, s_bad;
    __shared__ int s_count[kNff];
    if (threadIdx.x < 3) {
        s_lo[threadIdx.x] = 0xffffffffu;
        s_hi[threadIdx.x] = 0u;
    }
    if (threadIdx.x < kNff) s_count[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_mask = 0, s_bad = 0;
    __syncthreads();
    unsigned int lo[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, hi[3] = {0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 v = p[i];
        unsigned int o[3] = {f2o(v.x), f2o(v.y), f2o(v.z)};
        for (int k = 0; k < 3; ++k) {
            lo[k] = min(lo[k], o[k]);
            hi[k] = max(hi[k], o[k]);
        }
        if (!(isfinite(v.x) && isfinite(v.y) && isfinite(v.z))) atomicOr(&s_bad, 2u);
        if (ff_typed) {
            int t = __float_as_int(v.w);
            if (t <= kExv || t >= kNff) atomicOr(&s_bad, 1u);
            else {
                atomicOr(&s_mask, 1u << t);
                atomicAdd(&s_count[t], 1);
            }
        }
    }
    for (int k = 0; k < 3; ++k) {
        atomicMin(&s_lo[k], lo[k]);
        atomicMax(&s_hi[k], hi[k]);
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&st->lo[threadIdx.x], s_lo[threadIdx.x]);
        atomicMax(&st->hi[threadIdx.x], s_hi[threadIdx.x]);
    }
    if (threadIdx.x < kNff && s_count[threadIdx.x]) atomicAdd(&st->count[threadIdx.x], s_count[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicOr(&st->mask, s_mask);
        atomicOr(&st->bad, s_bad);
    }
}

__device__ __forceinline__ float o2f(unsigned int o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// max |p - c|^2 in double over the three point sets; non-negative doubles order like their bits
__global__ void radius_kernel(const float4* a, int na, const float4* w, int nw, const float4* x, int nx, PrepStats* st) {
    double c[3];
    for (int k = 0; k < 3; ++k) c[k] = 0.5 * ((double)o2f(st->lo[k]) + (double)o2f(st->hi[k]));
    double r2 = 0;
    const int n = na + nw + nx;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = i < na ? a[i] : (i < na + nw ? w[i - na] : x[i - na - nw]);
        const double dx = v.x - c[0], dy = v.y - c[1], dz = v.z - c[2];
        r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
    }
    for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    if ((threadIdx.x & 31) == 0 && r2 > 0) atomicMax(&st->r2, static_cast<unsigned long long>(__double_as_longlong(r2)));
}

__global__ void to_dense_kernel(const float4* in, float4* out, int n, const int32_t* ff_to_type) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 v = in[i];
        int t = __float_as_int(v.w);
        int d = (t > kExv && t < kNff) ? ff_to_type[t] : 0;
        v.w = __int_as_float(d);
        out[i] = v;
    }
}

__global__ void set_type_kernel(float4* p, int n, int32_t value) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i].w = __int_as_float(value);
}

}  // namespace

void census_launch(const float4* p, int n, int ff_typed, PrepStats* st, int sm_count, cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count * 2) blocks = sm_count * 2;
    census_kernel<<<blocks, 256, 0, s>>>(p, n, ff_typed, st);
}

void radius_launch(const float4* a, int na, const float4* w, int nw, const float4* x, int nx, PrepStats* st,
                   int sm_count, cudaStream_t s) {
    const long long n = (long long)na + nw + nx;
    if (n <= 0) return;
    long long blocks = (n + 255) / 256;
    if (blocks > sm_count * 2) blocks = sm_count * 2;
    radius_kernel<<<(int)blocks, 256, 0, s>>>(a, na, w, nw, x, nx, st);
}

void to_dense_launch(const float4* in, float4* out, int n, const int32_t* ff_to_type, int sm_count, cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count * 4) blocks = sm_count * 4;
    to_dense_kernel<<<blocks, 256, 0, s>>>(in, out, n, ff_to_type);
}

void set_type_launch(float4* p, int n, int32_t value, int sm_count, cudaStream_t s) {
    if (n <= 0) return;
    int blocks = (n + 255) / 256;
    if (blocks > sm_count * 4) blocks = sm_count * 4;
    set_type_kernel<<<blocks, 256, 0, s>>>(p, n, value);
}

// host-side inverse of f2o
float ordered_to_float(unsigned int o) {
    unsigned int u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

}  // namespace ausaxs_b200
