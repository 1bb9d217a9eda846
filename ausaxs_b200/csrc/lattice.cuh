// Pair-distance histogram of points on the integer lattice (grid excluded-volume dummies), by the
// autocorrelation of their occupancy (see lattice.cu).
#pragma once
#include "common.cuh"

namespace ausaxs_b200 {

// Occupancy of a point set on the integer lattice as bit lines along x: line (y, z) holds
// `words` u32 words, bit x set when a point sits at (lo_x + x, lo_y + y, lo_z + z).  Only the
// non-empty lines are stored (in (z, y) order); table[z * ly + y] is a line's index or -1.
struct LatticeGrid {
    int lo[3] = {0, 0, 0};
    int lx = 0, ly = 0, lz = 0, words = 0;
    int n_lines = 0;
    const uint32_t* lines = nullptr;  // [n_lines][words]
    const int32_t* table = nullptr;   // [lz][ly]
};

// Self pairs (i < j) of the lattice's points binned by the reference's rule into a single-row
// histogram: counts[bin] += pairs, dsum[bin] += pairs * (fixed-point in-bin offset), exactly the
// integers the pair kernel adds for the same points (a pair's bin and offset depend only on its
// squared distance, an integer).
struct LatticeLaunch {
    LatticeGrid G;
    int nbins;
    float inv_w, c, scale;
    unsigned long long* counts;    // [nbins]
    unsigned long long* dsum;      // [nbins] or null
    unsigned long long* overflow;  // pairs beyond the last bin
    unsigned long long* counter;   // work-item counter (zeroed before the launch)
    int n_items;                   // lz * (2 ly - 1) line offsets (dz >= 0) x kLatticeChunks z ranges
    const float4* pts;             // the points themselves, in the reference's loop order
    int n_pts;
    int tail_fix;                  // the two rounding rules differ at some squared offset: correct the
                                   // scalar-tail pairs (lattice_tail_kernel)
};

// Points per set below which the pair kernel is used for lattice points as well.
constexpr int kLatticeMinPoints = 1024;
constexpr int kLatticeMaxWords = 8;   // lines of up to 256 lattice cells along x
constexpr int kLatticeThreads = 512;  // lines of more than 128 cells; up to 128: 1024 threads
constexpr int kLatticeChunks = 4;     // z ranges per line offset (work items of one warp)

// Words per line of the kernel instantiation that serves a grid of `words` words (1, 2, 4 or 8).
inline int lattice_kernel_words(int words) { return words <= 2 ? words : (words <= 4 ? 4 : 8); }

// Dynamic shared memory of a launch (lines at the kernel's words per line, table, per-CTA histogram).
inline size_t lattice_smem_bytes(int n_lines, int words, int ly, int lz, int nbins) {
    size_t b = (size_t)n_lines * words * 4;
    b = (b + 15) & ~(size_t)15;
    b += ((size_t)ly * lz * 4 + 15) & ~(size_t)15;
    b += (size_t)(nbins + 1) * 16;
    return b + 64;
}

// Device scan of a point set (stats[0..2] minimum cell floor(v), [3..5] maximum, [6] non-zero when a
// coordinate is neither an integer nor an integer + 1/2 of magnitude < 2^20, [7] bit 2k: integers on
// axis k, bit 2k + 1: half-integers); stats must hold 8 ints.
void lattice_scan_launch(const float4* p, int n, int* stats, int sm_count, cudaStream_t s);
// Bit lines of the points (grid zeroed by the caller: ly * lz * words words), then the compact line
// store and the table; info[0] = lines, info[1] = non-zero when two points share a cell.
void lattice_build_launch(const float4* p, int n, const int lo[3], int lx, int ly, int lz, int words, uint32_t* grid,
                          uint32_t* lines, int32_t* table, int* info, int sm_count, cudaStream_t s);
// Whether the reference's two rounding rules (ties to even in its SIMD evaluators, ties away from
// zero in the scalar tail) bin every integer squared distance in [1, s2_max] alike at this inverse
// bin width; when they do not, lattice_launch also corrects the scalar-tail pairs.
bool lattice_rules_agree(long long s2_max, float inv_w);
// The lattice kernel, then (L.tail_fix) the scalar-tail correction.
void lattice_launch(const LatticeLaunch& L, int grid, size_t smem, cudaStream_t s);

}  // namespace ausaxs_b200
