// Point-set preparation kernels (see prep.cu).
#pragma once
#include <string.h>
#include "common.cuh"

namespace ausaxs_b200 {

struct PrepStats {
    unsigned int lo[3];  // order-preserving encodings of the bounding box
    unsigned int hi[3];
    unsigned int mask;   // bit t set: form-factor type t present
    unsigned int bad;    // bit 0: invalid form-factor type, bit 1: non-finite coordinate
    int count[kNff];     // atoms per form-factor type
    unsigned long long r2;  // bits of max |p - c|^2 (double) over every point, c = centre of the box
};

void census_launch(const float4* p, int n, int ff_typed, PrepStats* st, int sm_count, cudaStream_t s);
// After the census launches on the same stream: the radius of the points about the box centre
// (every pair distance is at most twice it).
void radius_launch(const float4* a, int na, const float4* w, int nw, const float4* x, int nx, PrepStats* st,
                   int sm_count, cudaStream_t s);
void to_dense_launch(const float4* in, float4* out, int n, const int32_t* ff_to_type, int sm_count, cudaStream_t s);
void set_type_launch(float4* p, int n, int32_t value, int sm_count, cudaStream_t s);
float ordered_to_float(unsigned int o);

}  // namespace ausaxs_b200
