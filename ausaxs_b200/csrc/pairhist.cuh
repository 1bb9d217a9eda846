// Pair-distance histogram kernels (the O(N^2) stage of the Debye hot path).
#pragma once
#include "common.cuh"

namespace ausaxs_b200 {

// Row selection of a pair job, by the histogram shape the reference increments.
enum RowMode : int32_t {
    kRowSingle = 0,  // one row (ww, xx, wx, and every Simple/weighted job)
    kRowPair = 1,    // [t_i][t_j] over dense atom types (increment_linear_index, CompactCoordinatesXYZFF.h:187-188)
    kRowOuter = 2    // [t_i] of the outer point (aw by atom type, HistogramManagerMTFFAvg.cpp:111-117; ax)
};

// One pass of pair binning: outer set A (index i) against inner set B (index j); self jobs visit
// only j > i (SimpleCalculator.h:117-141).  The host splits the pass into square tiles of
// kTile x kTile pairs; tiles of all jobs of a launch are numbered consecutively.
struct PairJob {
    const float4* A;
    const float4* B;
    int32_t na, nb;
    int32_t self;
    int32_t row_mode;
    int32_t types;        // dense type count T (kRowPair: rows = T*T, kRowOuter: rows = T)
    int32_t row_lo, row_hi;  // rows of this job kept by this pass (row-group split when the full set
                             // of rows does not fit on chip)
    int32_t nbins;        // bins on chip / in the global accumulators
    int32_t tiles_i, tiles_j;
    int64_t tile_begin;   // first global tile id of the job
    int64_t tile_count;
    float inv_w;          // float(1 / bin_width), the reference's multiplier
    float c;              // 1 / inv_w (float): bin pitch of the fixed-point offsets
    float scale;          // 2^20 / c
    unsigned long long* counts;  // [row_hi-row_lo][nbins] global pair counts (factor not applied)
    unsigned long long* dsum;    // [nbins] biased fixed-point offset sums, or null
    long long* wsum;             // [nbins] biased fixed-point weight-product sums, or null (weighted jobs):
                                 //         per pair rint(w_i w_j * wscale) + 2^30
    float wscale;                // unused (the launch-wide scale lives in device memory)
    // Where this job's pairs sit in the reference's loops, for its scalar-tail rule: outer point i's
    // row runs over inner indices [row_begin, tail_end) of the full point set, row_begin =
    // a_base + i + 1 when tail_from_outer (self loops) else 0, and the job's inner point j is point
    // b_base + j of that set.  A plain job: a_base = b_base = 0, tail_end = nb, tail_from_outer =
    // self.  A partial job (one body pair of a multi-body structure) keeps the full structure's rows.
    int32_t a_base, b_base, tail_end, tail_from_outer;
    // Multiplicity of every pair of the job (>= 1): its count, offset and weight contributions are
    // added mult times, as SimpleCalculator's scaling factor does (SimpleCalculator.h:291-330).
    int32_t mult;
};

struct PairLaunch {
    const PairJob* jobs;
    int32_t n_jobs;
    int64_t total_tiles;
    int32_t chunk;                  // tiles taken per grab from the global counter
    int32_t smem_rows;              // rows of the on-chip count array
    int32_t smem_bins;              // bins of the on-chip arrays (>= every job's nbins)
    unsigned long long* tile_counter;
    unsigned long long* overflow;   // pairs whose bin fell outside the job's nbins (bit 62: a bounded
                                    // wait of the kernel ran out)
    int32_t weighted;
    const float* wscale;            // device: 2^k with max|w_i w_j| * 2^k < 2^30 (weighted launches)
    int32_t dreg;                   // u64 offset sums in registers instead of shared memory (pairhist_dreg)
    int32_t stages;                 // staging buffers of inner tiles (set by pairhist_launch from the
                                    // shared memory it is given: 2 = the next tile's copy overlaps)
    float inv_w;                    // the inverse bin width every job of the launch shares (0: unknown)
    int32_t nr_sqrt;                // 1: the Newton-Raphson root (pair_sqrt_nr), set by pairhist_launch for
                                    // a width pair_sqrt_prepare verified (else the correctly rounded root);
                                    // 2: that, with a power-of-two inv_w fused into the bin rounding
    int32_t max_grabs;              // > 0: a CTA takes at most this many chunks and exits (the grid
                                    // must then cover the tiles: grid * max_grabs * chunk >= total);
                                    // bounded CTAs let the block scheduler interleave other launches
    int32_t groups;                 // 2: unweighted launches with shared-memory offset sums run tile
                                    // threads per CTA in two groups that split every tile's inner
                                    // points (pairhist_groups); 0 or 1: tile / kOuter threads
};

// Outer points per thread: a tile of `tile` points per side runs tile / kOuter threads.
constexpr int kOuter = 2;
inline int pairhist_threads(int tile) { return tile / kOuter; }

// Shared-memory budget of one CTA (opt-in maximum less the static allocations) and the footprint above
// which only one CTA fits on an SM.
constexpr size_t kPairSmemCap = 232448 - 1024;
constexpr size_t kPairSmemTwoPerSm = 233472 / 2 - 1024;
// Register-held offset sums cover bins [0, kDregBins): thread t holds bins t + k * threads.
constexpr int kDregBins = 4096;

// Bytes of dynamic shared memory of a launch's layout (pairhist_kernel): counts [rows][bins + 1]
// (the last column collects overflow), u64 offset sums (unless dreg: in registers), the u32 offset
// accumulator, weight sums (weighted), and `stages` buffers of `tile` inner points.
inline size_t pairhist_layout_bytes(int rows, int bins, bool weighted, int tile, bool dreg, int stages) {
    size_t pad = (size_t)bins + 1;
    size_t row = (pad * 4 + 15) & ~(size_t)15;
    size_t b = ((size_t)rows * pad * 4 + 15) & ~(size_t)15;  // u32 counts
    if (!dreg) b += (pad * 8 + 15) & ~(size_t)15;            // offset sums: u64
    b += row;                                                // u32 offset accumulator
    if (weighted) b += 2 * row;                              // weight sums (lo, hi)
    b += (size_t)stages * tile * 16;                         // inner tiles of points (16-byte aligned)
    return b + 64;
}

// The launch's footprint: double-buffered staging when it fits and costs no CTA per SM, else one buffer.
inline size_t pairhist_smem_bytes(int rows, int bins, bool weighted, int tile, bool dreg = false) {
    const size_t one = pairhist_layout_bytes(rows, bins, weighted, tile, dreg, 1);
    const size_t two = pairhist_layout_bytes(rows, bins, weighted, tile, dreg, 2);
    if (two > kPairSmemCap) return one;
    const int threads_cap = 2048 / pairhist_threads(tile);
    auto ctas = [threads_cap](size_t b) {
        const int by_smem = (int)(233472 / (b + 1024));
        return by_smem < threads_cap ? by_smem : threads_cap;
    };
    return ctas(two) >= ctas(one) ? two : one;
}

// Whether a launch keeps its u64 offset sums in registers: unweighted launches of at most kDregBins bins
// whose shared-memory layout holds the CTA to one per SM anyway (the register variant is compiled for
// one CTA per SM); the freed pad * 8 bytes let more count rows stay on chip.
inline bool pairhist_dreg(int rows, int bins, bool weighted, int tile) {
    return !weighted && bins <= kDregBins && pairhist_smem_bytes(rows, bins, weighted, tile) > kPairSmemTwoPerSm;
}

inline size_t pairhist_launch_smem(int rows, int bins, bool weighted, int tile) {
    return pairhist_smem_bytes(rows, bins, weighted, tile, pairhist_dreg(rows, bins, weighted, tile));
}

// Resident CTAs per SM of a launch with this footprint (the runtime's occupancy of the instantiation;
// groups as PairLaunch::groups).
int pairhist_ctas_per_sm(size_t smem, int tile, bool dreg, bool weighted, int groups = 1);

// Thread groups per CTA for a launch of `tiles` tiles: two groups (twice the threads on the same tile
// and shared memory) where one group per CTA would leave CTA slots without a tile (small structures:
// each tile then takes half the time) or would hold an SM to at most two CTAs (few warps per SM); one
// otherwise.
// Launches with weighted bins or register-held offset sums keep their own layouts (1).
int pairhist_groups(size_t smem, int tile, bool dreg, bool weighted, long long tiles, int sm_count);

// Rows of [rows][bins] counts that fit on chip for `tile`-point tiles (512 covers 256 as well).
inline int pairhist_max_rows(int bins, bool weighted, int tile = 512) {
    int r = 1;
    while (r < 4096 && pairhist_launch_smem(r + 1, bins, weighted, tile) <= kPairSmemCap) ++r;
    return r;
}

void pairhist_launch(const PairLaunch& L, int tile, int grid, size_t smem, cudaStream_t s);

// Exhaustive device check, once per process and inverse bin width, that pair_sqrt_nr bins every float
// squared distance below ((bins + 2) / inv_w)^2 exactly as the correctly rounded root does, under the
// reference's ties-to-even rule and its scalar tail's ties-away rule (synchronises the device; call it
// when planning, outside stream capture).  Launches over at most `bins` bins of a verified width then
// take the Newton-Raphson root.  Returns whether the width is verified.
bool pair_sqrt_prepare(float inv_w, int bins);

}  // namespace ausaxs_b200
