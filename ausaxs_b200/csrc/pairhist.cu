// Pair-distance histogram kernel: the O(N^2) stage of the Debye hot path on sm_100a.
//
// Replaces the reference's thread-pool drivers (include/core/hist/distance_calculator/
// SimpleCalculator.h:94-215 and the manager lambdas of HistogramManagerMTFFAvg.cpp:214-302,
// HistogramManagerMTFFExplicit.cpp:233-300, HistogramManagerMTFFGrid.cpp:68-159), their SIMD
// evaluators (CompactCoordinatesXYZW.h / XYZFF.h) and the thread-local histogram copies merged at
// the end (include/core/container/ThreadLocalWrapper.h:45-105).
//
// Design (B200):
//   * one persistent grid; CTAs take chunks of square tiles (TILE outer x TILE inner points) from a
//     global counter, over all jobs of the launch (aa, aw, ww, and ax, wx, xx for the grid model,
//     or every job of a batch of structures);
//   * each thread owns kOuter outer points in registers (lanes of a warp spread over the tile, so
//     that neighbouring points of a chain -- similar distances, same bins -- sit in different warps);
//     the inner tile is staged in shared memory by a 1D bulk copy (cp.async.bulk, mbarrier
//     completion; double-buffered when the layout allows, so the next tile's copy overlaps this
//     tile's pairs) and read as a broadcast float4 per inner point;
//   * every CTA keeps privatised histograms in shared memory: u32 counts per (row, bin), one u64
//     fixed-point sum of in-bin distance offsets per bin (the weighted bin centre), and for
//     weighted jobs one i64 fixed-point sum of weight products per bin; pairs beyond the last bin
//     land in one extra column per row and are counted as overflow when the CTA flushes;
//   * a CTA flushes its histograms to the global u64 accumulators when it moves to another job
//     (or before a 32-bit count could wrap), so the global traffic is one atomic per non-empty
//     on-chip bin per flush instead of one per pair.
// All accumulations are integer, so results do not depend on scheduling.
#include <cstring>
#include <map>
#include <mutex>

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

// ---------------------------------------------------------------------------------------------
// Bulk-copy staging (cp.async.bulk global -> shared with mbarrier transaction counts).  Every wait
// is bounded: after kWaitLimit polls the CTA records kWaitTimedOut in the launch's overflow word
// (the host then reports an error), waits (bounded) for its other copy in flight and stops.
// ---------------------------------------------------------------------------------------------
constexpr unsigned kWaitLimit = 1u << 24;
constexpr unsigned long long kWaitTimedOut = 1ull << 62;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(unsigned long long* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// thread 0: expect `bytes` on bar, then copy them (16-byte aligned, multiple of 16) into dst
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// orders this thread's generic-proxy accesses to shared memory before a later bulk copy into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// waits for phase `parity` of bar; false when the bound ran out
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    const uint32_t a = smem_addr(bar);
    for (unsigned it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32-bit add to a shared-memory word given by its shared-window byte address (no return value)
__device__ __forceinline__ void shared_red_add(uint32_t addr, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v));
}

// On-chip privatised histograms of one CTA.
//   counts   : u32 per (row, bin), one atomic per pair; column nbins of each row collects the pairs
//              beyond the last bin (overflow), counted at the flush.
//   offsets  : the in-bin distance offset of a pair is quantised to 16 bits (kResBits) and added
//              with a 32-bit atomic to dacc; every drain_segment<TILE>() inner points (at most 2^16
//              pairs per bin, so dacc cannot wrap) the threads drain dacc into the u64 sums d64
//              without atomics.  (A 64-bit shared-memory atomic costs about three times as much per
//              pair on sm_100a; this keeps one cheap 32-bit atomic per pair and an exact integer sum.)
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

// u64 offset sums held in registers (launches with DREG): thread t owns bins t + k * NT
template <int NT, bool DREG>
struct OffsetRegs {
    static constexpr int kSlots = DREG ? kDregBins / NT : 1;
    unsigned long long v[kSlots];
};

// dacc -> d64 (shared memory, or the thread's registers) for the bins of a job; callers synchronise
// before (atomics done) and after.
template <int NT, bool DREG>
__device__ __forceinline__ void drain_offsets(const Onchip& S, int nb, OffsetRegs<NT, DREG>& R) {
    if (DREG) {
#pragma unroll
        for (int k = 0; k < OffsetRegs<NT, DREG>::kSlots; ++k) {
            const int b = threadIdx.x + k * NT;
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
    for (int b = threadIdx.x; b < nb; b += NT) {
        uint32_t v = S.dacc[b];
        if (v) {
            S.d64[b] += v;
            S.dacc[b] = 0;
        }
    }
}

template <int NT, bool WEIGHTED, bool DREG>
__device__ __forceinline__ void flush_hist(const PairJob& J, const Onchip& S, OffsetRegs<NT, DREG>& R,
                                           unsigned long long* overflow) {
    __syncthreads();
    const int rows = J.row_hi - J.row_lo;
    const int nb = J.nbins;
    const int n = rows * nb;
    for (int idx = threadIdx.x; idx < n; idx += NT) {
        int r = idx / nb, b = idx - r * nb;
        uint32_t v = S.cnt[r * S.pad + b];
        if (v) {
            atomicAdd(&J.counts[static_cast<size_t>(r) * nb + b], static_cast<unsigned long long>(v) * J.mult);
            S.cnt[r * S.pad + b] = 0;
        }
    }
    // overflow column (bin nbins) of every row
    for (int r = threadIdx.x; r < rows; r += NT) {
        const uint32_t v = S.cnt[r * S.pad + nb];
        if (v) {
            atomicAdd(overflow, static_cast<unsigned long long>(v));
            S.cnt[r * S.pad + nb] = 0;
        }
    }
    if (DREG && J.dsum) {
#pragma unroll
        for (int k = 0; k < OffsetRegs<NT, DREG>::kSlots; ++k) {
            const int b = threadIdx.x + k * NT;
            if (b < nb && R.v[k]) atomicAdd(&J.dsum[b], R.v[k] * J.mult);
            R.v[k] = 0;
        }
    }
    for (int b = threadIdx.x; b < nb; b += NT) {
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

// Pairs of the thread's outer points against inner points [k0, k1) of the staged tile.  GENERAL
// handles the diagonal tiles of self jobs (j > i only), the tiles that contain scalar-tail
// partners and the last row of tiles (outer points beyond the set).  ROWS selects the count row:
// kRowsSingle, one row whose index is the bin; kRowsOffset, every row of the job is on chip and
// the staged inner points carry their row offset (inner type * pitch for pair rows, 0 for outer
// rows) in w; kRowsGeneric, a row group of a job whose rows do not all fit.
enum { kRowsSingle = 0, kRowsOffset = 1, kRowsGeneric = 2 };

struct Outer {
    float4 a;
    int i;           // index in the job's outer set
    int cbase;       // count index of bin 0 in its row (kRowsSingle / kRowsOffset), or its row base (generic)
    uint32_t caddr;  // kRowsSingle / kRowsOffset: shared byte address of its row's count of bin 0, less
                     // 4 * kMagicBits (so that 4 * (bits of the magic-rounded distance) lands on the bin)
    int ts;          // first inner index (local) that goes through the scalar evaluator
    bool active;
};

// The count and offset arrays are indexed with the bit pattern of the magic-rounded distance
// (kMagic + bin), their base pointers shifted by -kMagicBits.
template <bool GENERAL, bool WEIGHTED, int ROWS, int R, int NR, bool DSUM>
__device__ __forceinline__ void tile_pairs(const PairJob& J, const Onchip& S, const float4* s_pts, const Outer (&o)[R],
                                           int j0, int k0, int k1, bool diag, float wsc) {
    const float inv_w = J.inv_w, c = J.c, scale = J.scale;
    const float bin_limit = pair_bin_limit(J.nbins);  // kMagic + nbins: the overflow column
    const int rlo = J.row_lo, rhi = J.row_hi;
    const bool pair_rows = J.row_mode == kRowPair;
    constexpr bool do_d = DSUM;  // J.dsum != nullptr (a template argument: no branch per pair)
    const bool do_w = WEIGHTED && J.wsum != nullptr;
    uint32_t* const cnt = S.cnt - kMagicBits;
    // shared byte address of dacc[0] less 4 * kMagicBits (wrapping u32 arithmetic)
    const uint32_t dacc_addr = smem_addr(S.dacc) - 4u * static_cast<uint32_t>(kMagicBits);
#pragma unroll 4
    for (int jj = k0; jj < k1; ++jj) {
        const float4 b = s_pts[jj];
        const int j = j0 + jj;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if (GENERAL && (!o[k].active || (diag && j <= o[k].i))) continue;
            const float dx = __fsub_rn(o[k].a.x, b.x);
            const float dy = __fsub_rn(o[k].a.y, b.y);
            const float dz = __fsub_rn(o[k].a.z, b.z);
            float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
            bool tail = false;
            if (GENERAL) {
                tail = j >= o[k].ts;
                if (tail) s = __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
            }
            const float d = NR ? pair_sqrt_nr(s) : __fsqrt_rn(s);
            // rint(x), x = d inv_w, by the magic number, ties to even; distances past the last bin
            // (also NaN, inf and x >= 2^22) are clamped to the overflow column.  NR == 2: inv_w is a
            // power of two, so d inv_w is exact and one fused multiply-add rounds it
            float xm;
            if (NR == 2 && !GENERAL) {
                xm = fminf(__fmaf_rn(d, inv_w, kMagic), bin_limit);
            } else {
                const float x = __fmul_rn(d, inv_w);
                xm = fminf(__fadd_rn(x, kMagic), bin_limit);
                if (GENERAL && tail && __fsub_rn(x, __fsub_rn(xm, kMagic)) == 0.5f)
                    xm = fminf(__fadd_rn(xm, 1.0f), bin_limit);  // std::round: ties away from zero
            }
            const int xb = __float_as_int(xm);
            if (ROWS == kRowsSingle) {
                shared_red_add(o[k].caddr + (static_cast<uint32_t>(xb) << 2), 1u);
            } else if (ROWS == kRowsOffset) {
                // staged w: the inner point's row offset in bytes
                shared_red_add(o[k].caddr + static_cast<uint32_t>(__float_as_int(b.w)) + (static_cast<uint32_t>(xb) << 2), 1u);
            } else {
                // a row group: count the rows it keeps; the group with row 0 also carries the offset sums
                const int row = pair_rows ? o[k].cbase + __float_as_int(b.w) : o[k].cbase;
                if (row >= rlo && row < rhi) atomicAdd(&cnt[(row - rlo) * S.pad + xb], 1u);
            }
            if (do_d) {
                const float r = __fmaf_rn(-__fsub_rn(xm, kMagic), c, d);
                const float t = __fmaf_rn(r, scale, kMagic);  // rint(r * scale), one rounding
                shared_red_add(dacc_addr + (static_cast<uint32_t>(xb) << 2),
                               static_cast<uint32_t>(__float_as_int(t) - kMagicBits + kResBias));
            }
            if (do_w) {
                const float wp = __fmul_rn(o[k].a.w, b.w);
                const int wq = __float2int_rn(__fmul_rn(wp, wsc));  // |wq| <= 2^30
                add_carry(S.wlo, S.whi, xb - kMagicBits, static_cast<uint32_t>(wq + (1 << 30)));
            }
        }
    }
}

// G groups of NT / G threads split the inner points of a tile: group g takes inner points
// [g * TILE / G, (g + 1) * TILE / G); every group runs the same number of segments (the drains
// synchronise the CTA), and a segment spans NT * R pairs per inner point of every group, so
// drain_segment<NT * R>() keeps the 2^16-pairs-per-bin bound of the offset accumulators.
template <int NT, int R, bool WEIGHTED, bool DREG, int NR, int G>
__device__ __forceinline__ void run_segments(const PairJob& J, const Onchip& S, const float4* s_pts, const Outer (&o)[R],
                                             int j0, int jn, bool general, bool diag, float wsc,
                                             OffsetRegs<NT, DREG>& Rg) {
    constexpr int TILE = NT * R / G;
    constexpr int H = TILE / G;  // inner points per group
    constexpr int SEG = drain_segment<NT * R>();
    const bool single = J.row_mode == kRowSingle && J.row_lo == 0 && J.row_hi >= 1;
    const int full_rows = J.row_mode == kRowPair ? J.types * J.types : (J.row_mode == kRowOuter ? J.types : 1);
    const bool offset_rows = !single && J.row_lo == 0 && J.row_hi >= full_rows;
    const bool dsum = J.dsum != nullptr;
    const int g_lo = G > 1 ? static_cast<int>(threadIdx.x / (NT / G)) * H : 0;  // this group's first inner point
    const int g_hi = G > 1 ? min(jn, g_lo + H) : jn;
    const int span = G > 1 ? min(jn, H) : jn;  // group 0 has the most inner points: it sets the segment count
    for (int s0 = 0; s0 < span; s0 += SEG) {
        const int k0 = g_lo + s0;
        const int k1 = min(g_hi, k0 + SEG);
        if (general) {
            if (dsum) {
                if (single) tile_pairs<true, WEIGHTED, kRowsSingle, R, NR, true>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
                else if (offset_rows) tile_pairs<true, WEIGHTED, kRowsOffset, R, NR, true>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
                else tile_pairs<true, WEIGHTED, kRowsGeneric, R, NR, true>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
            } else {
                if (single) tile_pairs<true, WEIGHTED, kRowsSingle, R, NR, false>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
                else if (offset_rows) tile_pairs<true, WEIGHTED, kRowsOffset, R, NR, false>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
                else tile_pairs<true, WEIGHTED, kRowsGeneric, R, NR, false>(J, S, s_pts, o, j0, k0, k1, diag, wsc);
            }
        } else if (dsum) {
            if (single) tile_pairs<false, WEIGHTED, kRowsSingle, R, NR, true>(J, S, s_pts, o, j0, k0, k1, false, wsc);
            else if (offset_rows) tile_pairs<false, WEIGHTED, kRowsOffset, R, NR, true>(J, S, s_pts, o, j0, k0, k1, false, wsc);
            else tile_pairs<false, WEIGHTED, kRowsGeneric, R, NR, true>(J, S, s_pts, o, j0, k0, k1, false, wsc);
        } else {
            if (single) tile_pairs<false, WEIGHTED, kRowsSingle, R, NR, false>(J, S, s_pts, o, j0, k0, k1, false, wsc);
            else if (offset_rows) tile_pairs<false, WEIGHTED, kRowsOffset, R, NR, false>(J, S, s_pts, o, j0, k0, k1, false, wsc);
            else tile_pairs<false, WEIGHTED, kRowsGeneric, R, NR, false>(J, S, s_pts, o, j0, k0, k1, false, wsc);
        }
        if (dsum) {
            __syncthreads();
            drain_offsets<NT, DREG>(S, J.nbins, Rg);
            __syncthreads();
        }
    }
}

// DREG: the u64 offset sums live in registers (one CTA per SM; pairhist_dreg decides).  G > 1: the
// tile's side is NT * R / G points; G groups of NT / G threads share its outer points (R each) and
// split its inner points (run_segments), so a one-CTA layout keeps R = 2 outer points per thread
// (one staged inner point read per two pairs) with NT = 1024 threads on 1024-point tiles.
template <int NT, int R, bool WEIGHTED, bool DREG, int NR, int G>
__global__ void __launch_bounds__(NT, DREG ? 1 : (WEIGHTED ? (512 / NT > 1 ? 512 / NT : 1) : 1024 / NT)) pairhist_kernel(PairLaunch L) {
    constexpr int TILE = NT * R / G;
    constexpr int NTG = NT / G;  // threads per group
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ unsigned long long s_bar[2];
    __shared__ long long s_grab;
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
    // staging buffer b at stage0 + b * stage_pitch (one buffer: both indices name it)
    float4* const stage0 = reinterpret_cast<float4*>(smem + off);  // 16-byte aligned: every offset above is
    const int stage_pitch = L.stages > 1 ? TILE : 0;

    // zero the on-chip histograms once; drains and flushes keep them zero afterwards
    {
        uint32_t* z = reinterpret_cast<uint32_t*>(smem);
        const size_t words = off / 4;
        for (size_t k = threadIdx.x; k < words; k += NT) z[k] = 0;
    }
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    OffsetRegs<NT, DREG> Rg;
#pragma unroll
    for (int k = 0; k < OffsetRegs<NT, DREG>::kSlots; ++k) Rg.v[k] = 0;
    const float wsc = WEIGHTED ? *L.wscale : 0.f;
    // lanes of a warp take outer points NTG/32 apart; the warps of a group interleave
    const int tg = static_cast<int>(threadIdx.x % NTG);
    const int spread = (tg & 31) * (NTG / 32) + (tg >> 5);
    int cur = -1;
    long long pairs_since_flush = 0;
    unsigned phases = 0u;  // bit b: the parity of staging barrier b's next phase
    bool failed = false;

    // tile ids come in chunks from the global counter; the next tile id is known one tile ahead so
    // that its copy can be issued before the current tile is processed
    int grabs = 0;
    auto grab = [&]() -> long long {
        if (L.max_grabs > 0 && grabs >= L.max_grabs) return static_cast<long long>(L.total_tiles);  // block-uniform
        ++grabs;
        if (threadIdx.x == 0) s_grab = static_cast<long long>(atomicAdd(L.tile_counter, static_cast<unsigned long long>(L.chunk)));
        __syncthreads();
        const long long v = s_grab;
        __syncthreads();
        return v;
    };
    // inner points of tile g into staging buffer buf (thread 0 issues the copy)
    auto issue = [&](long long g, int buf) {
        if (threadIdx.x != 0) return;
        const int jb = find_job(L.jobs, L.n_jobs, g);
        const PairJob& J = L.jobs[jb];
        int ti, tj;
        tile_coords(J, g - J.tile_begin, ti, tj);
        const int j0 = tj * TILE;
        const int jn = min(TILE, J.nb - j0);
        bulk_load(stage0 + buf * stage_pitch, J.B + j0, static_cast<unsigned>(jn) * 16u, &s_bar[buf]);
    };

    long long g = grab();
    long long g_end = min(g + static_cast<long long>(L.chunk), static_cast<long long>(L.total_tiles));
    int buf = 0;
    if (g < L.total_tiles) issue(g, buf);
    while (g < L.total_tiles) {
        // the next tile: the rest of this chunk, else a new chunk
        long long gn = g + 1;
        if (gn >= g_end) {
            gn = grab();
            g_end = min(gn + static_cast<long long>(L.chunk), static_cast<long long>(L.total_tiles));
        }
        const bool prefetch = L.stages > 1 && gn < L.total_tiles;
        if (prefetch) issue(gn, buf ^ 1);  // buffer buf ^ 1 was released by the previous tile's final barrier

        const int jb = find_job(L.jobs, L.n_jobs, g);
        // u32 counts stay exact below 2^32 pairs per bin between flushes
        if (jb != cur || pairs_since_flush > (1ll << 31)) {
            if (cur >= 0) flush_hist<NT, WEIGHTED, DREG>(L.jobs[cur], S, Rg, L.overflow);
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

        // outer points and their row bases (overlaps the copy in flight)
        Outer o[R];
        const int row_begin_base = J.tail_from_outer ? J.a_base + 1 : 0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            o[k].i = ti * TILE + spread + k * NTG;
            o[k].active = o[k].i < J.na;
            o[k].a = o[k].active ? J.A[o[k].i] : make_float4(0.f, 0.f, 0.f, 0.f);
            const int ta = __float_as_int(o[k].a.w);
            const int rowbase = J.row_mode == kRowPair ? ta * J.types : (J.row_mode == kRowOuter ? ta : 0);
            o[k].cbase = single ? 0 : (offset_rows ? (rowbase - J.row_lo) * S.pad : rowbase);
            o[k].caddr = smem_addr(S.cnt) + 4u * static_cast<uint32_t>(o[k].cbase) - 4u * static_cast<uint32_t>(kMagicBits);
            const int row_begin = J.tail_from_outer ? row_begin_base + o[k].i : 0;
            o[k].ts = J.tail_end - ((J.tail_end - row_begin) & 3) - J.b_base;
        }

        const bool timed_out = !mbar_wait(&s_bar[buf], (phases >> buf) & 1u);
        phases ^= 1u << buf;
        if (__syncthreads_or(timed_out)) {  // block-uniform: every thread leaves together
            failed = true;
            if (threadIdx.x == 0) atomicOr(L.overflow, kWaitTimedOut);
            // the other buffer's copy, if one was issued, is waited for (bounded) before leaving
            if (prefetch) mbar_wait(&s_bar[buf ^ 1], (phases >> (buf ^ 1)) & 1u);
            break;
        }
        float4* s_pts = stage0 + buf * stage_pitch;
        if (offset_rows && J.row_mode == kRowPair) {
            // row offset of the inner point for jobs with every row on chip
            for (int k = threadIdx.x; k < jn; k += NT) s_pts[k].w = __int_as_float(__float_as_int(s_pts[k].w) * S.pad * 4);
            __syncthreads();
        } else if (offset_rows) {
            for (int k = threadIdx.x; k < jn; k += NT) s_pts[k].w = __int_as_float(0);
            __syncthreads();
        }
        pairs_since_flush += static_cast<long long>(TILE) * TILE;
        const bool diag = J.self && ti == tj;
        const bool has_tail = J.b_base + j0 + jn > J.tail_end - 3;  // scalar-tail partners: last 3 of a row
        const bool full = (ti + 1) * TILE <= J.na;
        const bool general = diag || has_tail || !full;
        run_segments<NT, R, WEIGHTED, DREG, NR, G>(J, S, s_pts, o, j0, jn, general, diag, wsc, Rg);
        fence_proxy_async();  // this thread's accesses to the buffer before the next bulk copy into it
        __syncthreads();      // every thread is done with the buffer
        if (!prefetch && gn < L.total_tiles) issue(gn, buf);
        else buf ^= 1;
        g = gn;
    }
    if (cur >= 0 && !failed) flush_hist<NT, WEIGHTED, DREG>(L.jobs[cur], S, Rg, L.overflow);
    if (!failed && threadIdx.x == 0) {
        mbar_inval(&s_bar[0]);
        mbar_inval(&s_bar[1]);
    }
}

template <int NT, int R, bool WEIGHTED, bool DREG, int NR, int G>
void launch_one(const PairLaunch& L, int grid, size_t smem, cudaStream_t s) {
    cudaFuncSetAttribute(pairhist_kernel<NT, R, WEIGHTED, DREG, NR, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    pairhist_kernel<NT, R, WEIGHTED, DREG, NR, G><<<grid, NT, smem, s>>>(L);
}

template <int NT, bool WEIGHTED, bool DREG, int G = 1>
void launch_nr(const PairLaunch& L, int grid, size_t smem, cudaStream_t s) {
    if (L.nr_sqrt == 2) launch_one<NT, kOuter, WEIGHTED, DREG, 2, G>(L, grid, smem, s);
    else if (L.nr_sqrt == 1) launch_one<NT, kOuter, WEIGHTED, DREG, 1, G>(L, grid, smem, s);
    else launch_one<NT, kOuter, WEIGHTED, DREG, 0, G>(L, grid, smem, s);
}

// Register-held offset sums mean a layout of one CTA per SM; with 1024-point tiles that CTA runs
// 1,024 threads in two groups that split the inner points (32 warps per SM instead of 16, still two
// outer points per thread), the shared memory unchanged.
template <int TILE>
void launch_tile(const PairLaunch& L, int grid, size_t smem, cudaStream_t s) {
    constexpr int NT = TILE / kOuter;
    // register-held offset sums exist for unweighted launches only (pairhist_dreg)
    if (L.weighted) launch_nr<NT, true, false>(L, grid, smem, s);
    else if (L.dreg && TILE == 1024) launch_nr<TILE, false, true, 2>(L, grid, smem, s);
    else if (L.dreg) launch_nr<NT, false, true>(L, grid, smem, s);
    else if (L.groups == 2) launch_nr<TILE, false, false, 2>(L, grid, smem, s);
    else launch_nr<NT, false, false>(L, grid, smem, s);
}

template <int NT, int R, bool WEIGHTED, bool DREG, int G = 1>
int occupancy_one(size_t smem) {
    // the root variants share the launch shape; the fewest resident CTAs of them bounds the launch
    auto k = pairhist_kernel<NT, R, WEIGHTED, DREG, 0, G>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, NT, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    for (auto k2 : {pairhist_kernel<NT, R, WEIGHTED, DREG, 1, G>, pairhist_kernel<NT, R, WEIGHTED, DREG, 2, G>}) {
        int n2 = 0;
        if (cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n2, k2, NT, smem) == cudaSuccess && n2 < n)
            n = n2;
    }
    cudaGetLastError();
    return n > 0 ? n : 1;
}

template <int TILE>
int occupancy_tile(size_t smem, bool weighted, bool dreg, int groups) {
    constexpr int NT = TILE / kOuter;
    if (weighted) return occupancy_one<NT, kOuter, true, false>(smem);
    if (dreg) return occupancy_one<NT, kOuter, false, true>(smem);
    if (groups == 2) return occupancy_one<TILE, kOuter, false, false, 2>(smem);
    return occupancy_one<NT, kOuter, false, false>(smem);
}

// ---------------------------------------------------------------------------------------------
// Verification of the Newton-Raphson root per inverse bin width (pair_sqrt_prepare)
// ---------------------------------------------------------------------------------------------
__global__ void sqrt_check_kernel(uint32_t hi_bits, float inv_w, unsigned long long* mismatches) {
    unsigned long long bad = 0;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < hi_bits; b += (uint64_t)gridDim.x * blockDim.x) {
        const float s = __uint_as_float(static_cast<uint32_t>(b));
        const float xa = __fmul_rn(__fsqrt_rn(s), inv_w), xb = __fmul_rn(pair_sqrt_nr(s), inv_w);
        // ties to even (the SIMD evaluators) and ties away from zero (the scalar tail)
        if (rintf(xa) != rintf(xb) || roundf(xa) != roundf(xb)) ++bad;
    }
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(mismatches, bad);
}

struct SqrtVerified {
    std::mutex m;
    std::map<uint32_t, int> bins;  // inverse bin width (bits) -> bins verified (0: failed)
};
SqrtVerified g_sqrt;

}  // namespace

int pairhist_ctas_per_sm(size_t smem, int tile, bool dreg, bool weighted, int groups) {
    if (tile == 1024 && dreg && !weighted) return occupancy_one<1024, kOuter, false, true, 2>(smem);
    if (tile == 1024) return occupancy_tile<1024>(smem, weighted, dreg, groups);
    if (tile == 256) return occupancy_tile<256>(smem, weighted, dreg, groups);
    return occupancy_tile<512>(smem, weighted, dreg, groups);
}

int pairhist_groups(size_t smem, int tile, bool dreg, bool weighted, long long tiles, int sm_count) {
    if (weighted || dreg) return 1;
    const int per_sm = pairhist_ctas_per_sm(smem, tile, false, false, 1);
    return (tiles < (long long)sm_count * per_sm || per_sm <= 2) ? 2 : 1;
}

bool pair_sqrt_prepare(float inv_w, int bins) {
    if (!(inv_w > 0) || bins <= 0) return false;
    const int want = bins < 8192 ? 8192 : bins;
    uint32_t key;
    std::memcpy(&key, &inv_w, 4);
    {
        std::lock_guard<std::mutex> lk(g_sqrt.m);
        auto it = g_sqrt.bins.find(key);
        if (it != g_sqrt.bins.end() && (it->second == 0 || it->second >= want)) return it->second >= bins;
    }
    // every float below the squared distance of bin want + 2 (the overflow clamp lies below it)
    const double dmax = (want + 2.0) / inv_w;
    const float s_max = static_cast<float>(dmax * dmax);
    uint32_t hi;
    std::memcpy(&hi, &s_max, 4);
    unsigned long long* d = nullptr;
    unsigned long long h = 1;
    bool ok = false;
    if (hi < 0x7f800000u && cudaMalloc(&d, sizeof(unsigned long long)) == cudaSuccess) {
        if (cudaMemset(d, 0, sizeof(unsigned long long)) == cudaSuccess) {
            sqrt_check_kernel<<<148 * 8, 256>>>(hi + 1, inv_w, d);
            ok = cudaMemcpy(&h, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost) == cudaSuccess && h == 0;
        }
        cudaFree(d);
    }
    cudaGetLastError();
    std::lock_guard<std::mutex> lk(g_sqrt.m);
    g_sqrt.bins[key] = ok ? want : 0;
    return ok && want >= bins;
}

void pairhist_launch(const PairLaunch& L0, int tile, int grid, size_t smem, cudaStream_t s) {
    PairLaunch L = L0;
    // the Newton-Raphson root where every job's width was verified for its bins (pair_sqrt_prepare)
    L.nr_sqrt = 0;
    {
        // the jobs live in device memory; the launch's bins and the width recorded with them decide
        std::lock_guard<std::mutex> lk(g_sqrt.m);
        uint32_t key;
        std::memcpy(&key, &L.inv_w, 4);
        auto it = g_sqrt.bins.find(key);
        L.nr_sqrt = (L.inv_w > 0 && it != g_sqrt.bins.end() && it->second >= L.smem_bins) ? 1 : 0;
        // a power-of-two inverse width (0.25 A bins): the product d inv_w is exact, so the rounding to
        // a bin fuses with it (one FFMA per pair instead of FMUL + FADD)
        int e = 0;
        if (L.nr_sqrt && std::frexp(L.inv_w, &e) == 0.5f) L.nr_sqrt = 2;
    }
    // double-buffered staging when the launch was given the room for it
    L.stages = smem >= pairhist_layout_bytes(L.smem_rows, L.smem_bins, L.weighted != 0, tile, L.dreg != 0, 2) ? 2 : 1;
    if (tile == 1024) launch_tile<1024>(L, grid, smem, s);
    else if (tile == 256) launch_tile<256>(L, grid, smem, s);
    else launch_tile<512>(L, grid, smem, s);
}

}  // namespace ausaxs_b200
