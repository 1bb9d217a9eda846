// Pair-distance histogram kernel: the O(N^2) stage of the Debye hot path on sm_100a.
//
// Replaces the reference's thread-pool drivers (include/core/hist/distance_calculator/
// SimpleCalculator.h:94-215 and the manager lambdas of HistogramManagerMTFFAvg.cpp:214-302,
// HistogramManagerMTFFExplicit.cpp:233-300, HistogramManagerMTFFGrid.cpp:68-159), their SIMD
// evaluators (CompactCoordinatesXYZW.h / XYZFF.h) and the thread-local histogram copies merged at
// the end (include/core/container/ThreadLocalWrapper.h:45-105).
//
// Design (B200):
//   * one persistent grid; CTAs take chunks of square tiles (kTile outer x kTile inner points)
//     from a global counter, over all jobs of the launch (aa, aw, ww, and ax, wx, xx for the grid
//     model, or every job of a batch of structures);
//   * each thread owns one outer point in registers; the inner tile is staged in shared memory
//     and read as a broadcast float4 per pair;
//   * every CTA keeps privatised histograms in shared memory: u32 counts per (row, bin), one u64
//     fixed-point sum of in-bin distance offsets per bin (the weighted bin centre), and for
//     weighted jobs one i64 fixed-point sum of weight products per bin;
//   * a CTA flushes its histograms to the global u64 accumulators when it moves to another job
//     (or before a 32-bit count could wrap), so the global traffic is one atomic per non-empty
//     on-chip bin per flush instead of one per pair.
// All accumulations are integer, so results do not depend on scheduling.
#include "pairhist.cuh"

namespace ausaxs_b200 {

namespace {

__device__ __forceinline__ int find_job(const PairJob* jobs, int n, long long g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile_begin <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Local tile id -> (ti, tj).  Self jobs enumerate the upper triangle (tj >= ti) row by row.
__device__ __forceinline__ void tile_coords(const PairJob& J, long long t, int& ti, int& tj) {
    if (!J.self) {
        ti = static_cast<int>(t / J.tiles_j);
        tj = static_cast<int>(t % J.tiles_j);
        return;
    }
    const long long T = J.tiles_i;
    double b = 2.0 * T + 1.0;
    long long r = static_cast<long long>((b - sqrt(b * b - 8.0 * static_cast<double>(t))) * 0.5);
    if (r < 0) r = 0;
    if (r > T - 1) r = T - 1;
    auto start = [T](long long x) { return x * T - x * (x - 1) / 2; };
    while (r > 0 && start(r) > t) --r;
    while (r + 1 < T && start(r + 1) <= t) ++r;
    ti = static_cast<int>(r);
    tj = static_cast<int>(r + (t - start(r)));
}

template <int TILE, bool WEIGHTED>
__device__ __forceinline__ void flush_hist(const PairJob& J, int pad, uint32_t* s_cnt, unsigned long long* s_dsum,
                                           long long* s_wsum) {
    __syncthreads();
    const int rows = J.row_hi - J.row_lo;
    const int nb = J.nbins;
    const int n = rows * nb;
    for (int idx = threadIdx.x; idx < n; idx += TILE) {
        int r = idx / nb, b = idx - r * nb;
        uint32_t v = s_cnt[r * pad + b];
        if (v) {
            atomicAdd(&J.counts[static_cast<size_t>(r) * nb + b], static_cast<unsigned long long>(v));
            s_cnt[r * pad + b] = 0;
        }
    }
    for (int b = threadIdx.x; b < nb; b += TILE) {
        if (J.dsum) {
            unsigned long long v = s_dsum[b];
            if (v) {
                atomicAdd(&J.dsum[b], v);
                s_dsum[b] = 0;
            }
        }
        if (WEIGHTED && J.wsum) {
            long long v = s_wsum[b];
            if (v) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&J.wsum[b]), static_cast<unsigned long long>(v));
                s_wsum[b] = 0;
            }
        }
    }
    __syncthreads();
}

template <int TILE, bool WEIGHTED>
__global__ void __launch_bounds__(TILE) pairhist_kernel(PairLaunch L) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int pad = L.smem_bins + 1;
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem);
    size_t off = (static_cast<size_t>(L.smem_rows) * pad * 4 + 15) & ~static_cast<size_t>(15);
    unsigned long long* s_dsum = reinterpret_cast<unsigned long long*>(smem + off);
    off += (static_cast<size_t>(pad) * 8 + 15) & ~static_cast<size_t>(15);
    long long* s_wsum = reinterpret_cast<long long*>(smem + off);
    if (WEIGHTED) off += (static_cast<size_t>(pad) * 8 + 15) & ~static_cast<size_t>(15);
    float4* s_pts = reinterpret_cast<float4*>(smem + off);  // 16-byte aligned: every offset above is
    __shared__ long long s_grab;

    // zero the on-chip histograms once; flushes keep them zero afterwards
    {
        uint32_t* z = reinterpret_cast<uint32_t*>(smem);
        size_t words = off / 4;
        for (size_t k = threadIdx.x; k < words; k += TILE) z[k] = 0;
    }
    __syncthreads();

    const float wsc = WEIGHTED ? *L.wscale : 0.f;
    int cur = -1;
    long long pairs_since_flush = 0;
    unsigned long long overflow = 0;

    for (;;) {
        if (threadIdx.x == 0) s_grab = static_cast<long long>(atomicAdd(L.tile_counter, static_cast<unsigned long long>(L.chunk)));
        __syncthreads();
        const long long g0 = s_grab;
        if (g0 >= L.total_tiles) break;
        const long long g1 = min(g0 + static_cast<long long>(L.chunk), static_cast<long long>(L.total_tiles));
        for (long long g = g0; g < g1; ++g) {
            const int jb = find_job(L.jobs, L.n_jobs, g);
            if (jb != cur || pairs_since_flush > (1ll << 31)) {
                if (cur >= 0) flush_hist<TILE, WEIGHTED>(L.jobs[cur], pad, s_cnt, s_dsum, s_wsum);
                cur = jb;
                pairs_since_flush = 0;
            }
            const PairJob& J = L.jobs[jb];
            int ti, tj;
            tile_coords(J, g - J.tile_begin, ti, tj);
            const int j0 = tj * TILE;
            const int jn = min(TILE, J.nb - j0);
            __syncthreads();  // previous tile done with s_pts
            if (threadIdx.x < jn) s_pts[threadIdx.x] = J.B[j0 + threadIdx.x];
            const int i = ti * TILE + threadIdx.x;
            const bool active = i < J.na;
            const float4 a = active ? J.A[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            __syncthreads();
            pairs_since_flush += static_cast<long long>(TILE) * TILE;

            const float inv_w = J.inv_w, c = J.c, scale = J.scale;
            const int nbins = J.nbins;
            const int rmode = J.row_mode, rlo = J.row_lo, rhi = J.row_hi;
            const bool diag = J.self && ti == tj;
            const int ts = tail_start(J.self ? i + 1 : 0, J.nb);
            const int rowbase = rmode == kRowPair ? __float_as_int(a.w) * J.types : (rmode == kRowOuter ? __float_as_int(a.w) : 0);
            const bool do_d = J.dsum != nullptr;
            const bool do_w = WEIGHTED && J.wsum != nullptr;
            if (!active) continue;
#pragma unroll 4
            for (int jj = 0; jj < jn; ++jj) {
                const float4 b = s_pts[jj];
                const int j = j0 + jj;
                if (diag && j <= i) continue;
                const PairBin p = pair_eval(a, b, inv_w, j >= ts);
                if (static_cast<unsigned>(p.bin) >= static_cast<unsigned>(nbins)) {
                    ++overflow;
                    continue;
                }
                const int row = rmode == kRowPair ? rowbase + __float_as_int(b.w) : rowbase;
                if (row >= rlo && row < rhi) atomicAdd(&s_cnt[(row - rlo) * pad + p.bin], 1u);
                if (do_d) atomicAdd(&s_dsum[p.bin], static_cast<unsigned long long>(pair_residual(p, c, scale)));
                if (do_w) {
                    const float wp = __fmul_rn(a.w, b.w);
                    const long long wq = __float2ll_rn(__fmul_rn(wp, wsc));
                    atomicAdd(reinterpret_cast<unsigned long long*>(&s_wsum[p.bin]), static_cast<unsigned long long>(wq));
                }
            }
        }
    }
    if (cur >= 0) flush_hist<TILE, WEIGHTED>(L.jobs[cur], pad, s_cnt, s_dsum, s_wsum);
    // warp-aggregated overflow report
    for (int o = 16; o > 0; o >>= 1) overflow += __shfl_xor_sync(0xffffffffu, overflow, o);
    if ((threadIdx.x & 31) == 0 && overflow) atomicAdd(L.overflow, overflow);
}

}  // namespace

void pairhist_launch(const PairLaunch& L, int tile, int grid, size_t smem, cudaStream_t s) {
    if (tile == 256) {
        if (L.weighted) {
            cudaFuncSetAttribute(pairhist_kernel<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            pairhist_kernel<256, true><<<grid, 256, smem, s>>>(L);
        } else {
            cudaFuncSetAttribute(pairhist_kernel<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            pairhist_kernel<256, false><<<grid, 256, smem, s>>>(L);
        }
    } else {
        if (L.weighted) {
            cudaFuncSetAttribute(pairhist_kernel<512, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            pairhist_kernel<512, true><<<grid, 512, smem, s>>>(L);
        } else {
            cudaFuncSetAttribute(pairhist_kernel<512, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            pairhist_kernel<512, false><<<grid, 512, smem, s>>>(L);
        }
    }
}

}  // namespace ausaxs_b200
