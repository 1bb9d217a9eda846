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

// On-chip privatised histograms of one CTA.
//   counts   : u32 per (row, bin), one atomic per pair.
//   offsets  : the in-bin distance offset of a pair is quantised to 16 bits (kResBits) and added
//              with a 32-bit atomic to dacc; every drain_segment<TILE>() inner points (at most 2^16 pairs per
//              bin, so dacc cannot wrap) the threads drain dacc into the u64 sums d64 without
//              atomics.  (A 64-bit shared-memory atomic costs about three times as much per pair on
//              sm_100a; this keeps one cheap 32-bit atomic per pair and an exact integer sum.)
//   weights  : weighted (Simple) jobs add rint(w_i w_j wscale) + 2^30 to wlo with exact carry
//              propagation into whi (the old value returned by the atomic detects the wrap).
struct Onchip {
    uint32_t* cnt;                // [rows][pad]
    uint32_t* dacc;               // [pad]
    unsigned long long* d64;      // [pad]
    uint32_t* wlo;                // [pad] (weighted launches)
    uint32_t* whi;                // [pad]
    int pad;
};

__device__ __forceinline__ void add_carry(uint32_t* lo, uint32_t* hi, int b, uint32_t v) {
    const uint32_t old = atomicAdd(&lo[b], v);
    if (old + v < old) atomicAdd(&hi[b], 1u);
}

// u64 offset sums held in registers (launches with DREG): thread t owns bins t + k * TILE
template <int TILE, bool DREG>
struct OffsetRegs {
    static constexpr int kSlots = DREG ? kDregBins / TILE : 1;
    unsigned long long v[kSlots];
};

// dacc -> d64 (shared memory, or the thread's registers) for the bins of a job; callers synchronise
// before (atomics done) and after.
template <int TILE, bool DREG>
__device__ __forceinline__ void drain_offsets(const Onchip& S, int nb, OffsetRegs<TILE, DREG>& R) {
    if (DREG) {
#pragma unroll
        for (int k = 0; k < OffsetRegs<TILE, DREG>::kSlots; ++k) {
            const int b = threadIdx.x + k * TILE;
            if (b < nb) {
                const uint32_t v = S.dacc[b];
                if (v) {
                    R.v[k] += v;
                    S.dacc[b] = 0;
                }
            }
        }
        return;
    }
    for (int b = threadIdx.x; b < nb; b += TILE) {
        uint32_t v = S.dacc[b];
        if (v) {
            S.d64[b] += v;
            S.dacc[b] = 0;
        }
    }
}

template <int TILE, bool WEIGHTED, bool DREG>
__device__ __forceinline__ void flush_hist(const PairJob& J, const Onchip& S, OffsetRegs<TILE, DREG>& R) {
    __syncthreads();
    const int rows = J.row_hi - J.row_lo;
    const int nb = J.nbins;
    const int n = rows * nb;
    for (int idx = threadIdx.x; idx < n; idx += TILE) {
        int r = idx / nb, b = idx - r * nb;
        uint32_t v = S.cnt[r * S.pad + b];
        if (v) {
            atomicAdd(&J.counts[static_cast<size_t>(r) * nb + b], static_cast<unsigned long long>(v) * J.mult);
            S.cnt[r * S.pad + b] = 0;
        }
    }
    if (DREG && J.dsum) {
#pragma unroll
        for (int k = 0; k < OffsetRegs<TILE, DREG>::kSlots; ++k) {
            const int b = threadIdx.x + k * TILE;
            if (b < nb && R.v[k]) atomicAdd(&J.dsum[b], R.v[k] * J.mult);
            R.v[k] = 0;
        }
    }
    for (int b = threadIdx.x; b < nb; b += TILE) {
        if (!DREG && J.dsum) {
            unsigned long long v = S.d64[b];
            if (v) {
                atomicAdd(&J.dsum[b], v * J.mult);
                S.d64[b] = 0;
            }
        }
        if (WEIGHTED && J.wsum) {
            unsigned long long v = (static_cast<unsigned long long>(S.whi[b]) << 32) | S.wlo[b];
            if (v) {
                atomicAdd(reinterpret_cast<unsigned long long*>(&J.wsum[b]), v * J.mult);
                S.wlo[b] = S.whi[b] = 0;
            }
        }
    }
    __syncthreads();
}

// Pairs of one outer point against inner points [k0, k1) of the staged tile.  GENERAL handles the
// diagonal tiles of self jobs (j > i only) and the tiles that contain scalar-tail partners.  ROWS
// selects the count row: kRowsSingle, one row whose index is the bin; kRowsOffset, every row of the
// job is on chip and the staged inner points carry their row offset (inner type * pitch for pair
// rows, 0 for outer rows) in w; kRowsGeneric, a row group of a job whose rows do not all fit.
enum { kRowsSingle = 0, kRowsOffset = 1, kRowsGeneric = 2 };

template <bool GENERAL, bool WEIGHTED, int ROWS>
__device__ __forceinline__ void tile_pairs(const PairJob& J, const Onchip& S, const float4* s_pts, const float4 a, int i,
                                           int j0, int k0, int k1, bool diag, float wsc, unsigned long long& overflow) {
    const float inv_w = J.inv_w, c = J.c, scale = J.scale;
    const unsigned nbins = static_cast<unsigned>(J.nbins);
    const float bin_limit = pair_bin_limit(J.nbins);
    const int rmode = J.row_mode, rlo = J.row_lo, rhi = J.row_hi;
    // first inner index (local) whose pair goes through the scalar evaluator: in the reference's
    // j-loops (SimpleCalculator.h:117-141, HistogramManagerMTFFAvg.cpp:216-232) the last
    // (row length mod 4) partners of each outer point do
    const int row_begin = J.tail_from_outer ? J.a_base + i + 1 : 0;
    const int ts = J.tail_end - ((J.tail_end - row_begin) & 3) - J.b_base;
    const int ta = __float_as_int(a.w);
    const bool pair_rows = rmode == kRowPair;
    const int rowbase = pair_rows ? ta * J.types : (rmode == kRowOuter ? ta : 0);
    const int cnt_base = (rowbase - rlo) * S.pad;  // kRowsOffset: + inner offset + bin
    const bool do_d = J.dsum != nullptr;
    const bool do_w = WEIGHTED && J.wsum != nullptr;
#pragma unroll 4
    for (int jj = k0; jj < k1; ++jj) {
        const float4 b = s_pts[jj];
        PairBin p;
        if (GENERAL) {
            const int j = j0 + jj;
            if (diag && j <= i) continue;
            p = pair_eval(a, b, inv_w, j >= ts);
            if (static_cast<unsigned>(p.bin) >= nbins) {
                ++overflow;
                continue;
            }
        } else if (!pair_eval_simd(a, b, inv_w, bin_limit, p)) {
            ++overflow;
            continue;
        }
        if (ROWS == kRowsSingle) {
            atomicAdd(&S.cnt[p.bin], 1u);
        } else if (ROWS == kRowsOffset) {
            atomicAdd(&S.cnt[cnt_base + __float_as_int(b.w) + p.bin], 1u);
        } else {
            const int row = pair_rows ? rowbase + __float_as_int(b.w) : rowbase;
            if (row >= rlo && row < rhi) atomicAdd(&S.cnt[(row - rlo) * S.pad + p.bin], 1u);
        }
        if (do_d) atomicAdd(&S.dacc[p.bin], pair_residual(p, c, scale));
        if (do_w) {
            const float wp = __fmul_rn(a.w, b.w);
            const int wq = __float2int_rn(__fmul_rn(wp, wsc));  // |wq| <= 2^30
            add_carry(S.wlo, S.whi, p.bin, static_cast<uint32_t>(wq + (1 << 30)));
        }
    }
}

// DREG: the u64 offset sums live in registers (one CTA per SM; pairhist_dreg decides)
template <int TILE, bool WEIGHTED, bool DREG>
__global__ void __launch_bounds__(TILE, DREG ? 1 : 1024 / TILE) pairhist_kernel(PairLaunch L) {
    extern __shared__ __align__(16) unsigned char smem[];
    Onchip S;
    S.pad = L.smem_bins + 1;
    const size_t w32 = (static_cast<size_t>(S.pad) * 4 + 15) & ~static_cast<size_t>(15);
    const size_t w64 = (static_cast<size_t>(S.pad) * 8 + 15) & ~static_cast<size_t>(15);
    size_t off = 0;
    S.cnt = reinterpret_cast<uint32_t*>(smem);
    off += (static_cast<size_t>(L.smem_rows) * S.pad * 4 + 15) & ~static_cast<size_t>(15);
    S.d64 = reinterpret_cast<unsigned long long*>(smem + off);
    if (!DREG) off += w64;
    S.dacc = reinterpret_cast<uint32_t*>(smem + off);
    off += w32;
    S.wlo = reinterpret_cast<uint32_t*>(smem + off);
    if (WEIGHTED) off += w32;
    S.whi = reinterpret_cast<uint32_t*>(smem + off);
    if (WEIGHTED) off += w32;
    float4* s_pts = reinterpret_cast<float4*>(smem + off);  // 16-byte aligned: every offset above is
    __shared__ long long s_grab;

    // zero the on-chip histograms once; drains and flushes keep them zero afterwards
    {
        uint32_t* z = reinterpret_cast<uint32_t*>(smem);
        size_t words = off / 4;
        for (size_t k = threadIdx.x; k < words; k += TILE) z[k] = 0;
    }
    __syncthreads();

    OffsetRegs<TILE, DREG> R;
#pragma unroll
    for (int k = 0; k < OffsetRegs<TILE, DREG>::kSlots; ++k) R.v[k] = 0;
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
            // u32 counts stay exact below 2^32 pairs per bin between flushes
            if (jb != cur || pairs_since_flush > (1ll << 31)) {
                if (cur >= 0) flush_hist<TILE, WEIGHTED, DREG>(L.jobs[cur], S, R);
                cur = jb;
                pairs_since_flush = 0;
            }
            const PairJob& J = L.jobs[jb];
            int ti, tj;
            tile_coords(J, g - J.tile_begin, ti, tj);
            const int j0 = tj * TILE;
            const int jn = min(TILE, J.nb - j0);
            const bool single = J.row_mode == kRowSingle && J.row_lo == 0 && J.row_hi >= 1;
            const int full_rows = J.row_mode == kRowPair ? J.types * J.types : (J.row_mode == kRowOuter ? J.types : 1);
            const bool offset_rows = !single && J.row_lo == 0 && J.row_hi >= full_rows;
            __syncthreads();  // previous tile done with s_pts
            if (threadIdx.x < jn) {
                float4 v = J.B[j0 + threadIdx.x];
                // row offset of the inner point for jobs with every row on chip
                if (offset_rows) v.w = __int_as_float(J.row_mode == kRowPair ? __float_as_int(v.w) * S.pad : 0);
                s_pts[threadIdx.x] = v;
            }
            const int i = ti * TILE + threadIdx.x;
            const bool active = i < J.na;
            const float4 a = active ? J.A[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            __syncthreads();
            pairs_since_flush += static_cast<long long>(TILE) * TILE;
            const bool diag = J.self && ti == tj;
            const bool has_tail = J.b_base + j0 + jn > J.tail_end - 3;  // scalar-tail partners: last 3 of a row
            const bool general = diag || has_tail;
            for (int k0 = 0; k0 < jn; k0 += drain_segment<TILE>()) {
                const int k1 = min(jn, k0 + drain_segment<TILE>());
                if (active) {
                    if (general) {
                        if (single) tile_pairs<true, WEIGHTED, kRowsSingle>(J, S, s_pts, a, i, j0, k0, k1, diag, wsc, overflow);
                        else if (offset_rows) tile_pairs<true, WEIGHTED, kRowsOffset>(J, S, s_pts, a, i, j0, k0, k1, diag, wsc, overflow);
                        else tile_pairs<true, WEIGHTED, kRowsGeneric>(J, S, s_pts, a, i, j0, k0, k1, diag, wsc, overflow);
                    } else {
                        if (single) tile_pairs<false, WEIGHTED, kRowsSingle>(J, S, s_pts, a, i, j0, k0, k1, false, wsc, overflow);
                        else if (offset_rows) tile_pairs<false, WEIGHTED, kRowsOffset>(J, S, s_pts, a, i, j0, k0, k1, false, wsc, overflow);
                        else tile_pairs<false, WEIGHTED, kRowsGeneric>(J, S, s_pts, a, i, j0, k0, k1, false, wsc, overflow);
                    }
                }
                if (J.dsum) {
                    __syncthreads();
                    drain_offsets<TILE, DREG>(S, J.nbins, R);
                    __syncthreads();
                }
            }
        }
    }
    if (cur >= 0) flush_hist<TILE, WEIGHTED, DREG>(L.jobs[cur], S, R);
    // warp-aggregated overflow report
    for (int o = 16; o > 0; o >>= 1) overflow += __shfl_xor_sync(0xffffffffu, overflow, o);
    if ((threadIdx.x & 31) == 0 && overflow) atomicAdd(L.overflow, overflow);
}

}  // namespace

namespace {
template <int TILE, bool WEIGHTED, bool DREG>
void launch_one(const PairLaunch& L, int grid, size_t smem, cudaStream_t s) {
    cudaFuncSetAttribute(pairhist_kernel<TILE, WEIGHTED, DREG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pairhist_kernel<TILE, WEIGHTED, DREG><<<grid, TILE, smem, s>>>(L);
}
}  // namespace

void pairhist_launch(const PairLaunch& L, int tile, int grid, size_t smem, cudaStream_t s) {
    // register-held offset sums exist for unweighted launches only (pairhist_dreg)
    if (tile == 1024) {
        if (L.weighted) launch_one<1024, true, false>(L, grid, smem, s);
        else if (L.dreg) launch_one<1024, false, true>(L, grid, smem, s);
        else launch_one<1024, false, false>(L, grid, smem, s);
    } else if (tile == 256) {
        if (L.weighted) launch_one<256, true, false>(L, grid, smem, s);
        else if (L.dreg) launch_one<256, false, true>(L, grid, smem, s);
        else launch_one<256, false, false>(L, grid, smem, s);
    } else {
        if (L.weighted) launch_one<512, true, false>(L, grid, smem, s);
        else if (L.dreg) launch_one<512, false, true>(L, grid, smem, s);
        else launch_one<512, false, false>(L, grid, smem, s);
    }
}

}  // namespace ausaxs_b200
