// Manager post-processing on the device: the part of calculate_all() after the pair loops.
//
// From the integer accumulators of the pair kernel this builds, in FP64, what the reference's
// managers return: factors, self-correlation terms, the excluded-volume rows (as marginals of the
// atom-atom rows), the Z_exv scaling, the truncation to max_bin, and the weighted distance axes.
//   HistogramManagerMT.cpp:23-75, SimpleCalculator.h:143-161           (Simple / weights)
//   HistogramManagerMTFFAvg.cpp:304-371                                (FFAvg)
//   HistogramManagerMTFFExplicit.cpp:303-345                           (FFExplicit)
//   HistogramManagerMTFFGrid.cpp:161-233                               (FFGrid)
//   WeightedDistribution1D.cpp:51-58, DistanceHistogram.cpp:30-47     (weighted axis)
#include "finalize.cuh"

namespace ausaxs_b200 {

namespace {

// Sum of factor * d over the pairs of one job in bin b, from its fixed-point offsets:
// d = b*c + r for every pair, r = (acc - n * bias) / scale.
__device__ __forceinline__ double dist_sum(const unsigned long long* ds, const unsigned long long n, int b, float c,
                                           float scale) {
    if (!ds || n == 0) return 0.0;
    long long resid = static_cast<long long>(ds[b]) - static_cast<long long>(n) * kResBias;
    return static_cast<double>(n) * b * static_cast<double>(c) + static_cast<double>(resid) / static_cast<double>(scale);
}

// WeightedDistribution1D::get_weighted_axis for one bin: mean distance, or the bin's lower value when empty.
__device__ __forceinline__ double weighted_bin(double dsum, double count, int b, double width) {
    unsigned int cnt = static_cast<unsigned int>(count);
    double dv = 0 + b * width;
    return (static_cast<double>(dsum == 0) * dv + dsum) / static_cast<double>((cnt == 0) + cnt);
}

__device__ void ff_maxbin_body(const FinalizeFF& F) {
    const int T = F.T;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(F.max_bin, 10);  // minimum size (HistogramManagerMT.cpp:48)
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < F.nb; b += gridDim.x * blockDim.x) {
        unsigned long long tot = 0;
        for (int r = 0; r < T * T; ++r) tot += 2ull * F.cnt_aa[static_cast<size_t>(r) * F.nb + b];
        for (int t = 0; t < T; ++t) tot += F.cnt_aw[static_cast<size_t>(t) * F.nb + b];
        tot += 2ull * F.cnt_ww[b];
        if (b == 0) tot += static_cast<unsigned long long>(F.n_a) + F.n_w;
        bool nz = tot != 0;
        if (F.kind == kKindGrid) {
            unsigned long long xx = 2ull * F.cnt_xx[b] + (b == 0 ? F.n_x : 0);
            nz = nz || xx != 0 || F.cnt_wx[b] != 0;
        }
        if (nz && b >= 10) atomicMax(F.max_bin, b + 1);
    }
}

__device__ void ff_rows_body(const FinalizeFF& F) {
    const int T = F.T;
    const int mb = *F.max_bin;
    const double width = (static_cast<double>(mb) * F.bin_width) / mb;  // Axis(0, mb*width, mb).width()
    const int R = ff_rows(T);
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < F.nb; b += gridDim.x * blockDim.x) {
        const size_t nb = F.nb;
        if (b >= mb) {
            for (int r = 0; r < R; ++r) F.H[r * nb + b] = 0;
            F.tot[b] = 0;
            F.d_axis[b] = 0;
            if (F.d_axis_ax) F.d_axis_ax[b] = 0;
            if (F.d_axis_xx) F.d_axis_xx[b] = 0;
            continue;
        }
        // atom-atom rows: factor 2, self terms (ff, ff, 0) += atoms of that type
        unsigned long long n_aa = 0, tot = 0;
        double xx_sum = 0;
        for (int ta = 0; ta < T; ++ta) {
            double ax_sum = 0;
            for (int tb = 0; tb < T; ++tb) {
                unsigned long long c = F.cnt_aa[static_cast<size_t>(ta * T + tb) * nb + b];
                n_aa += c;
                double v = 2.0 * static_cast<double>(c);
                if (b == 0 && ta == tb) v += F.type_count[ta];
                F.H[static_cast<size_t>(ta * T + tb) * nb + b] = v;
                ax_sum += 2.0 * static_cast<double>(c);
                tot += 2ull * c;
            }
            // [ff][exv] rows: every atom-atom pair also increments (ff_i, exv) with the lower-index
            // atom's type (HistogramManagerMTFFAvg.cpp:27-35), i.e. the marginal over ff_j
            double ax = 0;
            if (F.kind == kKindAvg) ax = ax_sum * F.z_exv;
            else if (F.kind == kKindGrid) ax = static_cast<double>(F.cnt_ax[static_cast<size_t>(ta) * nb + b]);
            F.H[static_cast<size_t>(T * T + ta) * nb + b] = ax;
            xx_sum += ax_sum;
        }
        if (b == 0) tot += static_cast<unsigned long long>(F.n_a);
        double xx = 0;
        // val * (Z * Z): the reference's release build hoists Z*Z (HistogramManagerMTFFAvg.cpp:361-362)
        if (F.kind == kKindAvg) xx = (xx_sum + (b == 0 ? F.n_a : 0)) * (F.z_exv * F.z_exv);
        else if (F.kind == kKindGrid) xx = 2.0 * static_cast<double>(F.cnt_xx[b]) + (b == 0 ? F.n_x : 0);
        F.H[static_cast<size_t>(T * T + T) * nb + b] = xx;
        // atom-water rows (factor 1) and their exv marginal
        unsigned long long n_aw = 0;
        for (int t = 0; t < T; ++t) {
            unsigned long long c = F.cnt_aw[static_cast<size_t>(t) * nb + b];
            n_aw += c;
            F.H[static_cast<size_t>(T * T + T + 1 + t) * nb + b] = static_cast<double>(c);
        }
        tot += n_aw;
        double wx = 0;
        if (F.kind == kKindAvg) wx = static_cast<double>(n_aw) * F.z_exv;
        else if (F.kind == kKindGrid) wx = static_cast<double>(F.cnt_wx[b]);
        F.H[static_cast<size_t>(T * T + 2 * T + 1) * nb + b] = wx;
        unsigned long long n_ww = F.cnt_ww[b];
        double ww = 2.0 * static_cast<double>(n_ww) + (b == 0 ? F.n_w : 0);
        F.H[static_cast<size_t>(T * T + 2 * T + 2) * nb + b] = ww;
        tot += 2ull * n_ww + (b == 0 ? static_cast<unsigned long long>(F.n_w) : 0ull);
        F.tot[b] = static_cast<double>(tot);

        // weighted axis of p_tot = aa(ff >= 1) + aw(ff >= 1) + ww, bin 0 pinned to 0
        if (F.weighted) {
            double ds = 2.0 * dist_sum(F.ds_aa, n_aa, b, F.c, F.scale) + dist_sum(F.ds_aw, n_aw, b, F.c, F.scale) +
                        2.0 * dist_sum(F.ds_ww, n_ww, b, F.c, F.scale);
            F.d_axis[b] = b == 0 ? 0.0 : weighted_bin(ds, static_cast<double>(tot), b, width);
        } else {
            F.d_axis[b] = b * width;
        }
        if (F.kind == kKindGrid) {
            // ax + wx share one axis, xx has its own; neither pins bin 0 (CompositeDistanceHistogramFFGrid.cpp:129-134)
            unsigned long long n_ax = 0;
            for (int t = 0; t < T; ++t) n_ax += F.cnt_ax[static_cast<size_t>(t) * nb + b];
            unsigned long long n_wx = F.cnt_wx[b];
            double ds_ax = dist_sum(F.ds_ax, n_ax, b, F.c, F.scale) + dist_sum(F.ds_wx, n_wx, b, F.c, F.scale);
            F.d_axis_ax[b] = weighted_bin(ds_ax, static_cast<double>(n_ax + n_wx), b, width);
            unsigned long long n_xx = F.cnt_xx[b];
            double ds_xx = 2.0 * dist_sum(F.ds_xx, n_xx, b, F.c, F.scale);
            F.d_axis_xx[b] = weighted_bin(ds_xx, 2.0 * n_xx + (b == 0 ? F.n_x : 0), b, width);
        }
    }
}

__global__ void ff_maxbin_kernel(FinalizeFF F) { ff_maxbin_body(F); }
__global__ void ff_rows_kernel(FinalizeFF F) { ff_rows_body(F); }
// batched: blockIdx.y selects the structure
__global__ void ff_maxbin_batch_kernel(const FinalizeFF* Fs) { ff_maxbin_body(Fs[blockIdx.y]); }
__global__ void ff_rows_batch_kernel(const FinalizeFF* Fs) { ff_rows_body(Fs[blockIdx.y]); }

// Expansion of the compact rows to the reference's [15][15] / [15] layouts, stride max_bin.
__global__ void ff_expand_kernel(FinalizeFF F, double* aa_out, double* aw_out) {
    const int T = F.T;
    const int mb = *F.max_bin;
    const size_t nb = F.nb;
    const int n = kNff * kNff * mb;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        int row = idx / mb, b = idx - row * mb;
        int f1 = row / kNff, f2 = row - f1 * kNff;
        double v = 0;
        int t1 = F.ff_to_type[f1], t2 = F.ff_to_type[f2];
        if (f1 != kExv && f2 != kExv) {
            if (t1 >= 0 && t2 >= 0) v = F.H[static_cast<size_t>(t1 * T + t2) * nb + b];
        } else if (f1 != kExv && f2 == kExv) {
            if (t1 >= 0 && F.kind != kKindExplicit) v = F.H[static_cast<size_t>(T * T + t1) * nb + b];
        } else if (f1 == kExv && f2 == kExv) {
            if (F.kind != kKindExplicit) v = F.H[static_cast<size_t>(T * T + T) * nb + b];
        }
        aa_out[idx] = v;
    }
    const int n2 = kNff * mb;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n2; idx += gridDim.x * blockDim.x) {
        int f = idx / mb, b = idx - f * mb;
        double v = 0;
        if (f == kExv) {
            if (F.kind != kKindExplicit) v = F.H[static_cast<size_t>(T * T + 2 * T + 1) * nb + b];
        } else if (F.ff_to_type[f] >= 0) {
            v = F.H[static_cast<size_t>(T * T + T + 1 + F.ff_to_type[f]) * nb + b];
        }
        aw_out[idx] = v;
    }
}

// ---- Simple / weighted (HistogramManagerMT) -------------------------------------------------

__global__ void weight_square_sum_kernel(const float4* p, int n, double* out) {
    double s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float w = p[i].w;
        s += static_cast<double>(__fmul_rn(w, w));  // float product, summed in double (SimpleCalculator.h:146-150)
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void weight_scale_kernel(const float4* a, int na, const float4* b, int nb, float* wscale) {
    // largest |w| over both sets; scale 2^k with (max|w|)^2 * 2^k <= 2^30
    __shared__ float s_max[32];
    float m = 0;
    for (int i = threadIdx.x; i < na; i += blockDim.x) m = fmaxf(m, fabsf(a[i].w));
    for (int i = threadIdx.x; i < nb; i += blockDim.x) m = fmaxf(m, fabsf(b[i].w));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mm = fmaxf(mm, s_max[k]);
        double p = static_cast<double>(mm) * mm;
        int e = 0;
        if (p > 0) frexp(p, &e);  // p < 2^e
        int k = 30 - e;
        if (k > 60) k = 60;
        *wscale = ldexpf(1.0f, k);
    }
}

// Weighted sum of one job in bin b: the pair kernel adds rint(w_i w_j * wscale) + 2^30 per pair
// (unsigned, wrapping); the bias is removed with n pairs counted in the bin.
__device__ __forceinline__ double weight_sum(const long long* w, const unsigned long long* n, int b, double inv) {
    unsigned long long raw = static_cast<unsigned long long>(w[b]) - n[b] * (1ull << 30);
    return static_cast<double>(static_cast<long long>(raw)) * inv;
}

__global__ void mt_maxbin_kernel(FinalizeMT F) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(F.max_bin, 10);  // minimum size (HistogramManagerMT.cpp:48)
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < F.nb; b += gridDim.x * blockDim.x) {
        double inv = 1.0 / static_cast<double>(*F.wscale);
        double v = 2.0 * weight_sum(F.w_aa, F.c_aa, b, inv) + 2.0 * weight_sum(F.w_ww, F.c_ww, b, inv) +
                   2.0 * weight_sum(F.w_aw, F.c_aw, b, inv);
        if (b == 0) v += *F.self_aa + *F.self_ww;
        if (v != 0 && b >= 10) atomicMax(F.max_bin, b + 1);
    }
}

__global__ void mt_rows_kernel(FinalizeMT F) {
    const int mb = *F.max_bin;
    const double width = (static_cast<double>(mb) * F.bin_width) / mb;
    const double inv = 1.0 / static_cast<double>(*F.wscale);
    const size_t nb = F.nb;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < F.nb; b += gridDim.x * blockDim.x) {
        if (b >= mb) {
            F.H[b] = F.H[nb + b] = F.H[2 * nb + b] = 0;
            F.tot[b] = 0;
            F.d_axis[b] = 0;
            continue;
        }
        double aa = 2.0 * weight_sum(F.w_aa, F.c_aa, b, inv);
        double aw = 2.0 * weight_sum(F.w_aw, F.c_aw, b, inv);
        double ww = 2.0 * weight_sum(F.w_ww, F.c_ww, b, inv);
        unsigned int c_aa = 2u * static_cast<unsigned int>(F.c_aa[b]);
        unsigned int c_aw = 2u * static_cast<unsigned int>(F.c_aw[b]);
        unsigned int c_ww = 2u * static_cast<unsigned int>(F.c_ww[b]);
        if (b == 0) {
            aa += *F.self_aa;
            ww += *F.self_ww;
            c_aa += static_cast<unsigned int>(*F.self_aa);
            c_ww += static_cast<unsigned int>(*F.self_ww);
        }
        F.H[b] = aa;
        F.H[nb + b] = aw;
        F.H[2 * nb + b] = ww;
        F.tot[b] = aa + ww + aw;
        if (F.weighted && b > 0) {
            double ds = 2.0 * dist_sum(F.ds_aa, F.c_aa[b], b, F.c, F.scale) + 2.0 * dist_sum(F.ds_ww, F.c_ww[b], b, F.c, F.scale) +
                        2.0 * dist_sum(F.ds_aw, F.c_aw[b], b, F.c, F.scale);
            F.d_axis[b] = weighted_bin(ds, static_cast<double>(c_aa + c_ww + c_aw), b, width);
        } else {
            F.d_axis[b] = b * width;
        }
        if (b == 0) F.d_axis[b] = 0;
    }
}

}  // namespace

void ff_finalize_launch(const FinalizeFF& F, cudaStream_t s) {
    int threads = 256;
    int blocks = (F.nb + threads - 1) / threads;
    ff_maxbin_kernel<<<blocks, threads, 0, s>>>(F);
    ff_rows_kernel<<<blocks, threads, 0, s>>>(F);
}

void ff_finalize_batch_launch(const FinalizeFF* Fs_dev, int n, int max_nb, cudaStream_t s) {
    int threads = 256;
    dim3 grid((max_nb + threads - 1) / threads, n);
    ff_maxbin_batch_kernel<<<grid, threads, 0, s>>>(Fs_dev);
    ff_rows_batch_kernel<<<grid, threads, 0, s>>>(Fs_dev);
}

void ff_expand_launch(const FinalizeFF& F, double* aa_out, double* aw_out, int nb_hint, cudaStream_t s) {
    int threads = 256;
    int blocks = (kNff * kNff * nb_hint + threads - 1) / threads;
    if (blocks > 2048) blocks = 2048;
    ff_expand_kernel<<<blocks, threads, 0, s>>>(F, aa_out, aw_out);
}

void weight_scale_launch(const float4* a, int na, const float4* b, int nb, float* wscale, cudaStream_t s) {
    weight_scale_kernel<<<1, 1024, 0, s>>>(a, na, b, nb, wscale);
}

void weight_square_sum_launch(const float4* p, int n, double* out, cudaStream_t s) {
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (blocks < 1) blocks = 1;
    weight_square_sum_kernel<<<blocks, 256, 0, s>>>(p, n, out);
}

void mt_finalize_launch(const FinalizeMT& F, cudaStream_t s) {
    int threads = 256;
    int blocks = (F.nb + threads - 1) / threads;
    mt_maxbin_kernel<<<blocks, threads, 0, s>>>(F);
    mt_rows_kernel<<<blocks, threads, 0, s>>>(F);
}

}  // namespace ausaxs_b200
