// Hydration shell on the device: what Molecule::generate_new_hydration() produces with the
// reference's default strategy, RadialHydration without culling
// (source/core/hydrate/generation/RadialHydration.cpp:43-206, GridBasedHydration.cpp:34-79).
//
// The reference tries 26 candidate positions around every atom, atom after atom, and accepts a
// candidate when its grid cell holds nothing but excluded volume and a collision check over 79 probe
// cells passes; an accepted water marks its cell and the empty cells within r_vdw(O) of it, which
// changes the outcome of later candidates.  The acceptance of candidate c therefore depends on the
// waters accepted before it, and adding a water can turn a later candidate either way (a blocked
// 1rh probe skips its direction's 3rh / 5rh terms, which may have been negative), so the sequential
// order has to be honoured.  Here it is resolved in rounds over all candidates at once:
//   * atom state of the cells (A_CENTER, A_AREA, VOLUME), kept across calls as the reference keeps its
//     grid: adding atoms sets their centre cells, the cells within r_vdw (A_AREA) and those within
//     rvol (VOLUME); removing atoms clears A_AREA and VOLUME within max(r_vdw, rvol) of each and
//     A_CENTER of its cell (Grid.cpp:293-400, SphericalExpander.h:27-76, 117-150).  The reference
//     sets A_AREA / VOLUME only on cells that are free at the time; setting them always gives the same
//     empty / excluded-volume / blocked classification, because a cell that was blocked when a bit
//     was withheld only becomes free again through a removal that clears that bit as well, so both
//     operations are order-free within a batch;
//   * candidates whose cell is outside the grid or statically blocked are rejected; the others are
//     undecided;
//   * each round, every undecided candidate w scatters its candidate index into the cells it would
//     mark (atomic minimum, "undecided" keys); every accepted one did so when it was accepted
//     ("accepted" keys).  For an undecided candidate c a probe cell is then blocked for sure
//     (statically, or by an accepted candidate before c), possibly blocked (by an undecided candidate
//     before c) or free; the collision check is evaluated over these three-valued cells as intervals
//     of the 1rh count and the score.  c is accepted when every outcome passes, rejected when every
//     outcome fails, and stays undecided otherwise.  Every decision is the sequential one, and the
//     earliest undecided candidate has no unknown cells, so every round decides at least one.
// Keys carry an epoch in their upper half (one per call for accepted keys, one per round for
// undecided keys), so the key grids are never cleared.  Waters come out in candidate order
// (atom * 26 + direction), the reference's order.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.cuh"
#include "guard.cuh"
#include "hydrate.cuh"

namespace ausaxs_b200 {
namespace {

constexpr double kRvol = 2.15;            // settings::grid::min_exv_radius (GridSettings.cpp:14)
constexpr double kRw = 1.71;              // Grid::get_hydration_radius(): r_vdw(O) (vdwTable.h:21)
constexpr double kShell = -0.35;          // settings::hydrate::shell_correction (MoleculeSettings.cpp:41)
constexpr double kMinScore = 0.25;        // settings::grid::detail::min_score (GridSettings.cpp:22)
constexpr double kNoiseSigma = 0.75;      // RadialHydration's default noise (RadialHydration.cpp:18-20)
// cell states as the reference's grid::detail::State bits (GridObj.h:17-24); waters are kept apart
constexpr uint8_t kVolume = 1, kACenter = 4, kAArea = 8, kBlock = kACenter | kAArea;
constexpr int kListThreads = 1024;        // one candidate per thread in the list passes
constexpr int kMaxRounds = 1 << 16;
constexpr int kBatch = 16;                // rounds between read-backs of the round counters

// constants::radius::get_vdw_radius(form_factor_t) (FormFactorType.h:173-192): H 1.1, C-family 1.96,
// N-family 1.79, O / OH 1.71, S / SH 2.06, OTHER (Ar) 1.88, UNKNOWN 0 A
__host__ __device__ inline double vdw(int ff) {
    switch (ff) {
        case 1: case 11: return 1.71;
        case 2: return 1.1;
        case 3: case 4: case 5: case 6: return 1.96;
        case 7: case 8: case 9: case 10: return 1.79;
        case 12: case 13: return 2.06;
        case 14: return 1.88;
        default: return 0.0;
    }
}

struct Dirs {
    double u[kHydDirections][3];
    int p1[kHydDirections][3], p3[kHydDirections][3], p5[kHydDirections][3];
};
__constant__ Dirs c_dirs;  // read with one index across the warp (a broadcast)
__device__ Dirs g_dirs;    // the same, read with a different index per lane: through the L1, since the
                           // constant cache serialises a warp's distinct addresses

// RadialHydration::prepare_rotations(8) (RadialHydration.cpp:73-141): theta, phi over one octant in
// steps of 2 pi / 8, reflected into the eight octants, components under 1e-5 zeroed, duplicates
// (distance < 1e-5) dropped in first-seen order; probe offsets (int)(round(k rh u) / width).
Dirs make_dirs() {
    Dirs D{};
    const double pi = 3.14159265358979323846, ang = 2 * pi / 8, rh = kRw + kShell;
    int n = 0;
    for (double theta = 0; theta <= pi * 0.5; theta += ang)
        for (double phi = 0; phi <= pi * 0.5; phi += ang) {
            const double x = std::cos(phi) * std::sin(theta), y = std::sin(phi) * std::sin(theta), z = std::cos(theta);
            const double s[8][3] = {{x, y, z}, {-x, y, z}, {x, -y, z}, {-x, -y, z},
                                    {x, y, -z}, {-x, y, -z}, {x, -y, -z}, {-x, -y, -z}};
            for (const auto& r : s) {
                double p[3] = {r[0], r[1], r[2]};
                for (double& v : p)
                    if (std::abs(v) < 1e-5) v = 0;
                bool present = false;
                for (int k = 0; k < n && !present; ++k) {
                    const double dx = D.u[k][0] - p[0], dy = D.u[k][1] - p[1], dz = D.u[k][2] - p[2];
                    present = std::sqrt(dx * dx + dy * dy + dz * dz) < 1e-5;
                }
                if (present) continue;
                if (n == kHydDirections) throw Error{AUSAXS_ERR_ARGUMENT, "hydration directions: more than 26"};
                for (int d = 0; d < 3; ++d) D.u[n][d] = p[d];
                ++n;
            }
        }
    if (n != kHydDirections) throw Error{AUSAXS_ERR_ARGUMENT, "hydration directions: fewer than 26"};
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            D.p1[i][d] = static_cast<int>(std::round(rh * D.u[i][d]) / 1.0);
            D.p3[i][d] = static_cast<int>(std::round(3 * rh * D.u[i][d]) / 1.0);
            D.p5[i][d] = static_cast<int>(std::round(5 * rh * D.u[i][d]) / 1.0);
        }
    return D;
}

struct HGrid {
    double gmin[3];
    int bins[3];
};

__device__ __forceinline__ size_t cell_at(const HGrid& G, int i, int j, int k) {
    return (static_cast<size_t>(i) * G.bins[1] + j) * G.bins[2] + k;
}
__device__ __forceinline__ bool in_grid(const HGrid& G, int i, int j, int k) {
    return i >= 0 && i < G.bins[0] && j >= 0 && j < G.bins[1] && k >= 0 && k < G.bins[2];
}
__device__ __forceinline__ void or_cell(uint8_t* cells, size_t q, uint8_t bit) {
    atomicOr(reinterpret_cast<unsigned int*>(cells) + (q >> 2), static_cast<unsigned int>(bit) << (8 * (q & 3)));
}
// squared distance from the centre of cell (i, j, k) to x, formed as the reference forms it:
// ((x_i - x)^2 + (y_j - y)^2) + (z_k - z)^2, each operation rounded on its own
__device__ __forceinline__ double dist2(const HGrid& G, int i, int j, int k, double x, double y, double z) {
    const double dx = __dsub_rn(__dadd_rn(G.gmin[0], (double)i), x);
    const double dy = __dsub_rn(__dadd_rn(G.gmin[1], (double)j), y);
    const double dz = __dsub_rn(__dadd_rn(G.gmin[2], (double)k), z);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// A_CENTER of every atom's cell; an atom outside the grid sets *err
__global__ void hyd_mark_centres(const double* __restrict__ xyz, long long n, HGrid G, uint8_t* cells, int* err) {
    for (long long a = blockIdx.x * (long long)blockDim.x + threadIdx.x; a < n; a += (long long)gridDim.x * blockDim.x) {
        const int i = (int)round(xyz[3 * a] - G.gmin[0]), j = (int)round(xyz[3 * a + 1] - G.gmin[1]),
                  k = (int)round(xyz[3 * a + 2] - G.gmin[2]);
        if (!in_grid(G, i, j, k)) {
            atomicExch(err, 1);
            continue;
        }
        or_cell(cells, cell_at(G, i, j, k), kACenter);
    }
}

// The atoms' spheres: one thread per (atom, x column, y column) of the box bin +- 3 (ceil(max(r, rvol))
// is 3 for every type); cells within r_vdw are blocked, those within rvol excluded volume.
constexpr int kSpan = 7;
__global__ void hyd_mark_spheres(const double* __restrict__ xyz, const int32_t* __restrict__ ff, long long n, HGrid G,
                                 uint8_t* cells) {
    const long long total = n * kSpan * kSpan;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long a = t / (kSpan * kSpan);
        const int col = (int)(t - a * kSpan * kSpan);
        const double x = xyz[3 * a], y = xyz[3 * a + 1], z = xyz[3 * a + 2];
        const double rv = vdw(ff[a]);
        const double rv2 = rv * rv, rvol2 = kRvol * kRvol;
        const int br = (int)ceil(fmax(rv, kRvol));
        const int di = col / kSpan - kSpan / 2, dj = col % kSpan - kSpan / 2;
        if (di < -br || di > br || dj < -br || dj > br) continue;
        const int bi = (int)round(x - G.gmin[0]), bj = (int)round(y - G.gmin[1]), bk = (int)round(z - G.gmin[2]);
        const int i = bi + di, j = bj + dj;
        if (i < 0 || i >= G.bins[0] || j < 0 || j >= G.bins[1]) continue;
        for (int k = max(bk - br, 0); k < min(bk + br + 1, G.bins[2]); ++k) {
            const double d = dist2(G, i, j, k, x, y, z);
            if (d <= rv2) or_cell(cells, cell_at(G, i, j, k), kAArea);
            else if (d <= rvol2) or_cell(cells, cell_at(G, i, j, k), kVolume);
        }
    }
}

__device__ __forceinline__ void and_cell(uint8_t* cells, size_t q, uint8_t keep) {
    atomicAnd(reinterpret_cast<unsigned int*>(cells) + (q >> 2), ~(static_cast<unsigned int>(~keep & 0xffu) << (8 * (q & 3))));
}

// Grid::remove of atoms at their current (old) positions: A_CENTER of each atom's cell cleared, and
// A_AREA / VOLUME of the cells within max(r_vdw, rvol) (the atom deflation, SphericalExpander.h:117-150)
__global__ void hyd_remove(const double* __restrict__ xyz, const int32_t* __restrict__ ff, long long n, HGrid G,
                           uint8_t* cells, int* err) {
    const long long total = n * kSpan * kSpan;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long a = t / (kSpan * kSpan);
        const int col = (int)(t - a * kSpan * kSpan);
        const double x = xyz[3 * a], y = xyz[3 * a + 1], z = xyz[3 * a + 2];
        const double rmax = fmax(vdw(ff[a]), kRvol), rmax2 = rmax * rmax;
        const int br = (int)ceil(rmax);
        const int bi = (int)round(x - G.gmin[0]), bj = (int)round(y - G.gmin[1]), bk = (int)round(z - G.gmin[2]);
        if (col == 0) {
            if (in_grid(G, bi, bj, bk)) and_cell(cells, cell_at(G, bi, bj, bk), (uint8_t)~kACenter);
            else atomicExch(err, 1);
        }
        const int di = col / kSpan - kSpan / 2, dj = col % kSpan - kSpan / 2;
        if (di < -br || di > br || dj < -br || dj > br) continue;
        const int i = bi + di, j = bj + dj;
        if (i < 0 || i >= G.bins[0] || j < 0 || j >= G.bins[1]) continue;
        for (int k = max(bk - br, 0); k < min(bk + br + 1, G.bins[2]); ++k)
            if (dist2(G, i, j, k, x, y, z) <= rmax2) and_cell(cells, cell_at(G, i, j, k), (uint8_t)~(kAArea | kVolume));
    }
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    // SplitMix64 (S. Vigna): a 64-bit counter-based mixer
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
// one Gaussian draw per (candidate, component) by the Box-Muller transform of two mixed counters
__device__ __forceinline__ double gauss(unsigned long long seed, long long c, int d) {
    const unsigned long long z1 = splitmix64(seed ^ (0x9e3779b97f4a7c15ull * (3ull * (unsigned long long)c + d + 1)));
    const unsigned long long z2 = splitmix64(z1);
    const double u1 = (double)((z1 >> 11) + 1) * 0x1p-53, u2 = (double)(z2 >> 11) * 0x1p-53;
    return kNoiseSigma * sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

struct Cand {
    double x[3];
    int b[3];
    bool keep;
};
// candidate c = atom * 26 + direction: x = fma(u, r_vdw + rh, atom + noise) (the reference build
// contracts atom + u reff + noise so), its cell, and whether it survives the static tests
__device__ __forceinline__ Cand candidate(long long c, const double* __restrict__ xyz, const int32_t* __restrict__ ff,
                                          const double* __restrict__ noise, unsigned long long seed, const HGrid& G,
                                          const uint8_t* __restrict__ cells) {
    Cand K;
    const long long a = c / kHydDirections;
    const int r = (int)(c - a * kHydDirections);
    const double reff = vdw(ff[a]) + (kRw + kShell);
    bool valid = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double nz = noise ? noise[3 * c + d] : (seed ? gauss(seed, c, d) : 0.0);
        K.x[d] = fma(__ldg(&g_dirs.u[r][d]), reff, __dadd_rn(xyz[3 * a + d], nz));
        K.b[d] = (int)round(K.x[d] - G.gmin[d]);
        valid = valid && K.b[d] >= 0 && K.b[d] < G.bins[d];
    }
    K.keep = valid && !(cells[cell_at(G, K.b[0], K.b[1], K.b[2])] & kBlock);
    return K;
}

// The collision check against the atoms alone, every other cell counted as possibly blocked: true when
// the candidate fails whatever the waters before it do (three or more 1rh probes on atoms, or a score
// that cannot exceed min_score * 3 * 26).  Reads the cell bytes only.
__device__ __forceinline__ bool fails_on_atoms(const int b[3], const HGrid& G, const uint8_t* __restrict__ cells) {
    int inside = 0, smax = 0;
#pragma unroll 2
    for (int i = 0; i < kHydDirections; ++i) {
        int q1[3], q3[3], q5[3];
        bool oob3 = false, oob5 = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            q1[d] = min(max(b[d] + c_dirs.p1[i][d], 0), G.bins[d] - 1);
            q3[d] = b[d] + c_dirs.p3[i][d];
            q5[d] = b[d] + c_dirs.p5[i][d];
            oob3 = oob3 || q3[d] < 0 || q3[d] >= G.bins[d];
            oob5 = oob5 || q5[d] < 0 || q5[d] >= G.bins[d];
        }
        const uint8_t s1 = cells[cell_at(G, q1[0], q1[1], q1[2])];
        const uint8_t s3 = oob3 ? 0 : cells[cell_at(G, q3[0], q3[1], q3[2])];
        const uint8_t s5 = oob5 ? 0 : cells[cell_at(G, q5[0], q5[1], q5[2])];
        if (s1 & kBlock) {
            ++inside;
            continue;
        }
        int ghi;
        if (oob3) ghi = 2;
        else if (s3 & kBlock) ghi = -2;
        else ghi = 2 + (oob5 ? 1 : ((s5 & kBlock) ? -1 : 0));
        smax += max(ghi, 0);
    }
    return inside >= 3 || smax <= kMinScore * 3 * kHydDirections;
}

__global__ void hyd_count(long long n_cand, const double* xyz, const int32_t* ff, const double* noise,
                          unsigned long long seed, HGrid G, const uint8_t* cells, uint8_t* flags,
                          unsigned int* block_counts) {
    const long long c = blockIdx.x * (long long)kListThreads + threadIdx.x;
    bool keep = false;
    if (c < n_cand) {
        const Cand K = candidate(c, xyz, ff, noise, seed, G, cells);
        keep = K.keep && !fails_on_atoms(K.b, G, cells);
        flags[c] = keep;
    }
    const int n = __syncthreads_count(keep);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = (unsigned int)n;
}

// exclusive scan of the block counts in one block; the total goes to *total
__global__ void hyd_scan(unsigned int* counts, int n, unsigned long long* total) {
    __shared__ unsigned long long carry;
    __shared__ unsigned int warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const unsigned int v = t < n ? counts[t] : 0u;
        unsigned int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31) >= o) x += y;
        }
        if ((threadIdx.x & 31) == 31) warp_sums[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x < 32) {
            const int nw = blockDim.x >> 5;
            unsigned int w = threadIdx.x < nw ? warp_sums[threadIdx.x] : 0u;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int y = __shfl_up_sync(0xffffffffu, w, o);
                if (threadIdx.x >= o) w += y;
            }
            if (threadIdx.x < nw) warp_sums[threadIdx.x] = w;
        }
        __syncthreads();
        const unsigned int warp_prefix = (threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5) - 1] : 0u;
        const unsigned long long excl = carry + warp_prefix + x - v;
        const unsigned int block_total = warp_sums[(blockDim.x >> 5) - 1];
        __syncthreads();
        if (t < n) counts[t] = (unsigned int)excl;
        if (threadIdx.x == 0) carry += block_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// position of this thread's flagged item among the block's flagged items, in thread order
__device__ __forceinline__ unsigned int block_rank(bool flag, unsigned int* warp_base) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned int ballot = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int acc = 0;
        for (int w = 0; w < kListThreads / 32; ++w) {
            const unsigned int c = warp_base[w];
            warp_base[w] = acc;
            acc += c;
        }
    }
    __syncthreads();
    return warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
}

struct List {
    double* x;            // [3][cap]
    int4* b;              // cell (i, j, k) and candidate index
    int8_t* state;        // 0 undecided, 1 accepted, -1 rejected
    unsigned int* active[2];
    long long cap;
};

__global__ void hyd_write(long long n_cand, const double* xyz, const int32_t* ff, const double* noise,
                          unsigned long long seed, HGrid G, const uint8_t* cells, const uint8_t* flags,
                          const unsigned int* offsets, List L) {
    __shared__ unsigned int warp_base[kListThreads / 32];
    const long long c = blockIdx.x * (long long)kListThreads + threadIdx.x;
    Cand K{};
    const bool keep = c < n_cand && flags[c];
    if (keep) K = candidate(c, xyz, ff, noise, seed, G, cells);
    const unsigned int rank = block_rank(keep, warp_base);
    if (!keep) return;
    const long long e = (long long)offsets[blockIdx.x] + rank;
    L.x[e] = K.x[0];
    L.x[L.cap + e] = K.x[1];
    L.x[2 * L.cap + e] = K.x[2];
    L.b[e] = make_int4(K.b[0], K.b[1], K.b[2], (int)c);
    L.state[e] = 0;
    L.active[0][e] = (unsigned int)e;
}

__device__ __forceinline__ unsigned long long key_of(uint32_t hi, int cand) {
    return ((unsigned long long)hi << 32) | (unsigned int)cand;
}

// The cells a water at x in cell b marks (Grid::add(water, expand = true), Grid.cpp:332-370 with
// SphericalExpander.h:78-115): its own cell, and the empty cells of the box b +- ceil(r_vdw(O)) = 2
// whose centre lies within r_vdw(O) of x.  Column (di, dj) of the box, all of its k.
constexpr int kWBox = 5;
template <typename F>
__device__ __forceinline__ void water_marks_column(const HGrid& G, const uint8_t* cells, const double* x, int4 b, int di,
                                                   int dj, F&& mark) {
    const int i = b.x + di, j = b.y + dj;
    if (i < 0 || i >= G.bins[0] || j < 0 || j >= G.bins[1]) return;
    const double rw2 = kRw * kRw;
    for (int k = max(b.z - 2, 0); k < min(b.z + 3, G.bins[2]); ++k) {
        const size_t q = cell_at(G, i, j, k);
        if ((di == 0 && dj == 0 && k == b.z) || (cells[q] == 0 && dist2(G, i, j, k, x[0], x[1], x[2]) <= rw2)) mark(q);
    }
}

__global__ void hyd_scatter(List L, const unsigned int* __restrict__ active, const unsigned long long* __restrict__ n_active,
                            HGrid G, const uint8_t* __restrict__ cells, unsigned long long* keys_und, uint32_t und_hi) {
    const long long n = (long long)*n_active * (kWBox * kWBox);
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long a = t / (kWBox * kWBox);
        const int col = (int)(t - a * kWBox * kWBox);
        const unsigned int e = active[a];
        const int4 b = L.b[e];
        const double x[3] = {L.x[e], L.x[L.cap + e], L.x[2 * L.cap + e]};
        const unsigned long long key = key_of(und_hi, b.w);
        water_marks_column(G, cells, x, b, col / kWBox - 2, col % kWBox - 2,
                           [&](size_t q) { atomicMin(keys_und + q, key); });
    }
}

enum : int { kFree = 0, kBlocked = 1, kUnknown = 2 };

// A probe cell's three values for candidate c, from its state byte and the two key words (all loaded
// at once): blocked by an atom or by a water accepted before c, possibly blocked by an undecided
// candidate before c, or free.
struct ProbeData {
    uint8_t st;
    unsigned long long acc, und;
};
__device__ __forceinline__ ProbeData probe_load(size_t q, const uint8_t* cells, const unsigned long long* keys_acc,
                                                const unsigned long long* keys_und) {
    return {__ldcg(cells + q), __ldcg(keys_acc + q), __ldcg(keys_und + q)};
}
__device__ __forceinline__ int probe_value(const ProbeData& p, int c, uint32_t acc_hi, uint32_t und_hi) {
    if (p.st & kBlock) return kBlocked;
    if ((uint32_t)(p.acc >> 32) == acc_hi && (int)(uint32_t)p.acc < c) return kBlocked;
    if ((uint32_t)(p.und >> 32) == und_hi && (int)(uint32_t)p.und < c) return kUnknown;
    return kFree;
}

// One warp per undecided candidate: lane i < 26 evaluates direction i of collision_check
// (RadialHydration.cpp:143-205) over three-valued cells, giving bounds of its 1rh count and score
// terms; lane 26 reads the candidate's own cell.  The warp sums the bounds; c is accepted when
// every outcome passes (own cell free, at most 2 blocked 1rh probes, score > min_score * 3 * 26),
// rejected when every outcome fails, and otherwise goes to the next round's list.  The marks of an
// accepted candidate (into the accepted keys) or of one that stays undecided (into the other array of
// undecided keys, read by the next round) are written by 25 lanes, one box column each.
__global__ void __launch_bounds__(256) hyd_evaluate(List L, const unsigned int* __restrict__ active,
                                                   const unsigned long long* __restrict__ n_active, unsigned int* next,
                                                   unsigned long long* n_next, HGrid G, const uint8_t* __restrict__ cells,
                                                   unsigned long long* keys_acc,
                                                   const unsigned long long* __restrict__ keys_und,
                                                   unsigned long long* keys_und_next, uint32_t acc_hi, uint32_t und_hi,
                                                   uint32_t und_hi_next) {
    const long long n = (long long)*n_active;
    const int lane = threadIdx.x & 31;
    const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
    const double min_points = kMinScore * 3 * kHydDirections;
    for (long long t = warp; t < n; t += warps) {
        const unsigned int e = active[t];
        const int4 b = L.b[e];
        const int c = b.w;
        int imin = 0, imax = 0, smin = 0, smax = 0, own = kFree;
        if (lane < kHydDirections) {
            int q1[3], q3[3], q5[3];
            bool oob3 = false, oob5 = false;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const int bd = d == 0 ? b.x : (d == 1 ? b.y : b.z);
                q1[d] = min(max(bd + __ldg(&g_dirs.p1[lane][d]), 0), G.bins[d] - 1);
                q3[d] = bd + __ldg(&g_dirs.p3[lane][d]);
                q5[d] = bd + __ldg(&g_dirs.p5[lane][d]);
                oob3 = oob3 || q3[d] < 0 || q3[d] >= G.bins[d];
                oob5 = oob5 || q5[d] < 0 || q5[d] >= G.bins[d];
            }
            // all probes of the direction at once (the 3rh / 5rh ones are read only inside the grid)
            const ProbeData d1 = probe_load(cell_at(G, q1[0], q1[1], q1[2]), cells, keys_acc, keys_und);
            ProbeData d3{0, ~0ull, ~0ull}, d5{0, ~0ull, ~0ull};
            if (!oob3) d3 = probe_load(cell_at(G, q3[0], q3[1], q3[2]), cells, keys_acc, keys_und);
            if (!oob5) d5 = probe_load(cell_at(G, q5[0], q5[1], q5[2]), cells, keys_acc, keys_und);
            const int s1 = probe_value(d1, c, acc_hi, und_hi);
            // the direction's 3rh / 5rh terms
            int glo, ghi;
            if (oob3) {
                glo = ghi = 2;
            } else {
                const int s3 = probe_value(d3, c, acc_hi, und_hi);
                int hlo, hhi;
                if (oob5) {
                    hlo = hhi = 1;
                } else {
                    const int s5 = probe_value(d5, c, acc_hi, und_hi);
                    hlo = s5 == kFree ? 0 : -1;
                    hhi = s5 == kBlocked ? -1 : 0;
                }
                if (s3 == kBlocked) glo = ghi = -2;
                else if (s3 == kFree) glo = 2 + hlo, ghi = 2 + hhi;
                else glo = -2, ghi = 2 + hhi;
            }
            if (s1 == kBlocked) {
                imin = imax = 1;
            } else if (s1 == kFree) {
                smin = glo, smax = ghi;
            } else {  // blocked (inside + 1, no terms) or free
                imax = 1;
                smin = min(glo, 0);
                smax = max(ghi, 0);
            }
        } else if (lane == kHydDirections) {
            own = probe_value(probe_load(cell_at(G, b.x, b.y, b.z), cells, keys_acc, keys_und), c, acc_hi, und_hi);
        }
        imin = __reduce_add_sync(0xffffffffu, imin);
        imax = __reduce_add_sync(0xffffffffu, imax);
        smin = __reduce_add_sync(0xffffffffu, smin);
        smax = __reduce_add_sync(0xffffffffu, smax);
        own = __shfl_sync(0xffffffffu, own, kHydDirections);
        int verdict;
        if (own == kBlocked) {
            verdict = -1;
        } else {
            const bool pass_sure = own == kFree && imax <= 2 && smin > min_points;
            const bool fail_sure = imin >= 3 || smax <= min_points;
            verdict = pass_sure ? 1 : (fail_sure ? -1 : 0);
        }
        if (verdict == 0) {
            if (lane == 0) next[atomicAdd(n_next, 1ull)] = e;
        } else if (lane == 0) {
            L.state[e] = (int8_t)verdict;
        }
        if (verdict != -1 && lane < kWBox * kWBox) {
            // accepted: its marks for every later reader; still undecided: its marks for the next round
            const double x[3] = {L.x[e], L.x[L.cap + e], L.x[2 * L.cap + e]};
            unsigned long long* keys = verdict == 1 ? keys_acc : keys_und_next;
            const unsigned long long key = key_of(verdict == 1 ? acc_hi : und_hi_next, c);
            water_marks_column(G, cells, x, b, lane / kWBox - 2, lane % kWBox - 2,
                               [&](size_t q) { atomicMin(keys + q, key); });
        }
    }
}

__global__ void hyd_count_accepted(const List L, const unsigned long long* __restrict__ n_list, unsigned int* block_counts) {
    const long long e = blockIdx.x * (long long)kListThreads + threadIdx.x;
    const bool acc = e < (long long)*n_list && L.state[e] == 1;
    const int n = __syncthreads_count(acc);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = (unsigned int)n;
}

__global__ void hyd_write_accepted(const List L, const unsigned long long* __restrict__ n_list,
                                   const unsigned int* offsets, double* waters, long long* cands) {
    __shared__ unsigned int warp_base[kListThreads / 32];
    const long long e = blockIdx.x * (long long)kListThreads + threadIdx.x;
    const bool acc = e < (long long)*n_list && L.state[e] == 1;
    const unsigned int rank = block_rank(acc, warp_base);
    if (!acc) return;
    const long long o = (long long)offsets[blockIdx.x] + rank;
    waters[3 * o] = L.x[e];
    waters[3 * o + 1] = L.x[L.cap + e];
    waters[3 * o + 2] = L.x[2 * L.cap + e];
    cands[o] = L.b[e].w;
}

}  // namespace

void hydrate_axes(const double* xyz, long long n, double gmin[3], int bins[3]) {
    // Grid(bodies) keeps the running box in a Vector3 deduced from {0, 0, 0}, i.e. of int
    // (Grid.cpp:36): every extent that widens it is truncated toward zero, and diff is an int
    int mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    for (long long a = 0; a < n; ++a)
        for (int d = 0; d < 3; ++d) {
            if (xyz[3 * a + d] < mn[d]) mn[d] = (int)xyz[3 * a + d];
            if (xyz[3 * a + d] > mx[d]) mx[d] = (int)xyz[3 * a + d];
        }
    const int diff[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    const double scaling = (diff[0] < 50 || diff[1] < 50 || diff[2] < 50) ? 1.0 : 0.25;
    const double margin = 2.14 + kRw + kShell + 3.0;  // r_vdw(P) + r_vdw(O) + shell correction + 3 cells
    for (int d = 0; d < 3; ++d) {
        const double e = std::max(0.5 * diff[d] * scaling, margin);
        gmin[d] = std::floor(mn[d] - e - 1.0);
        const double gmax = std::ceil(mx[d] + e + 1.0);
        bins[d] = (int)((gmax - gmin[d]) / 1.0);
    }
}

namespace {
HGrid to_grid(const double gmin[3], const int bins[3]) {
    HGrid G{};
    for (int d = 0; d < 3; ++d) G.gmin[d] = gmin[d], G.bins[d] = bins[d];
    return G;
}
size_t cell_count(const int bins[3]) { return (size_t)bins[0] * bins[1] * bins[2]; }
}  // namespace

void hydration_cells_check(const double gmin[3], const int bins[3]) {
    if (bins[0] <= 0 || bins[1] <= 0 || bins[2] <= 0) throw Error{AUSAXS_ERR_ARGUMENT, "empty hydration grid"};
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(gmin[d])) throw Error{AUSAXS_ERR_ARGUMENT, "invalid hydration grid axes"};
    if (cell_count(bins) >= ((size_t)1 << 34)) throw Error{AUSAXS_ERR_CAPACITY, "hydration grid of 2^34 cells or more"};
}

void hydration_add(Ctx& C, uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms, const int32_t* ff,
                   long long n, int* err) {
    if (n <= 0) return;
    const HGrid G = to_grid(gmin, bins);
    const int threads = 256;
    const int bc = (int)std::max(1LL, std::min((n + threads - 1) / threads, (long long)C.sm_count * 8));
    hyd_mark_centres<<<bc, threads, 0, C.stream>>>(atoms, n, G, cells, err);
    C.check_launch("hydration centres");
    const long long cols = n * kSpan * kSpan;
    const int bs = (int)std::max(1LL, std::min((cols + threads - 1) / threads, (long long)C.sm_count * 16));
    hyd_mark_spheres<<<bs, threads, 0, C.stream>>>(atoms, ff, n, G, cells);
    C.check_launch("hydration spheres");
}

void hydration_remove(Ctx& C, uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms,
                      const int32_t* ff, long long n, int* err) {
    if (n <= 0) return;
    const HGrid G = to_grid(gmin, bins);
    const int threads = 256;
    const long long cols = n * kSpan * kSpan;
    const int bs = (int)std::max(1LL, std::min((cols + threads - 1) / threads, (long long)C.sm_count * 16));
    hyd_remove<<<bs, threads, 0, C.stream>>>(atoms, ff, n, G, cells, err);
    C.check_launch("hydration removal");
}

void Hydrator::generate(Ctx& C, const uint8_t* cells, const double gmin[3], const int bins[3], const double* atoms,
                        const int32_t* ff, long long n, const double* noise, unsigned long long seed) {
    cudaStream_t s = C.stream;
    count = survivors = 0;
    rounds = 0;
    hydration_cells_check(gmin, bins);
    const size_t ncells = cell_count(bins);
    const long long n_cand = n * kHydDirections;
    if (n_cand >= INT_MAX) throw Error{AUSAXS_ERR_CAPACITY, "too many atoms for one hydration call"};
    static thread_local int dirs_device = -1;
    if (dirs_device != C.device) {
        const Dirs D = make_dirs();
        AUSAXS_CUDA(cudaMemcpyToSymbol(c_dirs, &D, sizeof(D)));
        AUSAXS_CUDA(cudaMemcpyToSymbol(g_dirs, &D, sizeof(D)));
        dirs_device = C.device;
    }
    const HGrid G = to_grid(gmin, bins);
    // key grids: accepted, and two of undecided (round r reads one, writes the next round's into the other)
    if (key_cells < ncells) {
        keys.ensure(align_up(3 * ncells * 8, 256));
        AUSAXS_CUDA(cudaMemsetAsync(keys.p, 0xff, 3 * ncells * 8, s));
        key_cells = ncells;
        call_epoch = round_epoch = 0;
    }
    if (call_epoch > 0xfff00000u || round_epoch > 0xfff00000u) {
        AUSAXS_CUDA(cudaMemsetAsync(keys.p, 0xff, 3 * key_cells * 8, s));
        call_epoch = round_epoch = 0;
    }
    unsigned long long* keys_acc = keys.as<unsigned long long>();
    unsigned long long* keys_und[2] = {keys_acc + key_cells, keys_acc + 2 * key_cells};
    const uint32_t acc_hi = 0xffffffffu - (++call_epoch);
    const long long cap = std::max(1LL, n_cand);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align_up(bytes, 256);
        return o;
    };
    const size_t o_x = take(3 * cap * 8), o_b = take(cap * 16), o_state = take(cap), o_a0 = take(cap * 4),
                 o_a1 = take(cap * 4);
    list.ensure(off);
    List L{list.as<double>(o_x), list.as<int4>(o_b), list.as<int8_t>(o_state),
           {list.as<unsigned int>(o_a0), list.as<unsigned int>(o_a1)}, cap};
    const long long nblocks = std::max(1LL, (n_cand + kListThreads - 1) / kListThreads);
    off = 0;
    const size_t o_counts = take(nblocks * 4), o_total = take(8), o_rounds = take((kMaxRounds + 1) * 8),
                 o_acc_total = take(8), o_flags = take(cap);
    off_waters = take(3 * cap * 8);
    off_cands = take(cap * 8);
    work.ensure(off);
    unsigned int* counts = work.as<unsigned int>(o_counts);
    unsigned long long* total = work.as<unsigned long long>(o_total);
    unsigned long long* round_n = work.as<unsigned long long>(o_rounds);
    unsigned long long* acc_total = work.as<unsigned long long>(o_acc_total);
    uint8_t* flags = work.as<uint8_t>(o_flags);

    cudaEvent_t ev;
    C.time_begin(5, &ev);
    AUSAXS_CUDA(cudaMemsetAsync(total, 0, 8, s));
    if (n > 0) {
        hyd_count<<<(unsigned)nblocks, kListThreads, 0, s>>>(n_cand, atoms, ff, noise, seed, G, cells, flags, counts);
        C.check_launch("hydration candidates");
        hyd_scan<<<1, 1024, 0, s>>>(counts, (int)nblocks, total);
        C.check_launch("hydration scan");
        hyd_write<<<(unsigned)nblocks, kListThreads, 0, s>>>(n_cand, atoms, ff, noise, seed, G, cells, flags, counts, L);
        C.check_launch("hydration list");
    }
    // the first round's undecided keys: every listed candidate
    const int grid_rounds = C.sm_count * 8;
    const int threads = 256;
    uint32_t epoch = ++round_epoch;
    if (n > 0) {
        hyd_scatter<<<grid_rounds, threads, 0, s>>>(L, L.active[0], total, G, cells, keys_und[0], 0xffffffffu - epoch);
        C.check_launch("hydration scatter");
    }
    // rounds, in batches between read-backs of the counters of undecided candidates
    std::vector<unsigned long long> h(kBatch);
    unsigned long long left = 0;
    C.time_end(5, ev);
    AUSAXS_CUDA(cudaMemcpyAsync(&left, total, 8, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    survivors = (long long)left;
    int r = 0;
    while (left > 0) {
        if (r + kBatch > kMaxRounds) throw Error{AUSAXS_ERR_CAPACITY, "hydration rounds exceed their bound"};
        C.time_begin(5, &ev);
        AUSAXS_CUDA(cudaMemsetAsync(round_n + r + 1, 0, kBatch * 8, s));
        for (int k = 0; k < kBatch; ++k, ++r) {
            const unsigned long long* n_in = r == 0 ? total : round_n + r;
            const uint32_t next_epoch = ++round_epoch;
            hyd_evaluate<<<grid_rounds, threads, 0, s>>>(L, L.active[r & 1], n_in, L.active[(r + 1) & 1], round_n + r + 1, G,
                                                      cells, keys_acc, keys_und[r & 1], keys_und[(r + 1) & 1], acc_hi,
                                                      0xffffffffu - epoch, 0xffffffffu - next_epoch);
            C.check_launch("hydration round");
            epoch = next_epoch;
        }
        C.time_end(5, ev);
        AUSAXS_CUDA(cudaMemcpyAsync(h.data(), round_n + r - kBatch + 1, kBatch * 8, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaStreamSynchronize(s));
        left = h[kBatch - 1];
        if (left == 0) {
            int used = r - kBatch;
            for (int k = 0; k < kBatch; ++k) {
                ++used;
                if (h[k] == 0) break;
            }
            rounds = used;
        }
    }
    // the accepted candidates in candidate order
    C.time_begin(5, &ev);
    if (survivors > 0) {
        const long long nlist = (survivors + kListThreads - 1) / kListThreads;
        hyd_count_accepted<<<(unsigned)nlist, kListThreads, 0, s>>>(L, total, counts);
        C.check_launch("hydration count");
        hyd_scan<<<1, 1024, 0, s>>>(counts, (int)nlist, acc_total);
        C.check_launch("hydration scan");
        hyd_write_accepted<<<(unsigned)nlist, kListThreads, 0, s>>>(L, total, counts, work.as<double>(off_waters),
                                                                 work.as<long long>(off_cands));
        C.check_launch("hydration write");
    } else {
        AUSAXS_CUDA(cudaMemsetAsync(acc_total, 0, 8, s));
    }
    C.time_end(5, ev);
    unsigned long long res = 0;
    AUSAXS_CUDA(cudaMemcpyAsync(&res, acc_total, 8, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    count = (long long)res;
}

void Hydrator::run(Ctx& C, const double* atoms, const int32_t* ff, long long n, const double gmin[3], const int bins[3],
                   const double* noise, unsigned long long seed) {
    hydration_cells_check(gmin, bins);
    const size_t ncells = cell_count(bins);
    cells.ensure(align_up(ncells, 256) + 256);
    int* err = cells.as<int>(align_up(ncells, 256));
    cudaEvent_t ev;
    C.time_begin(5, &ev);
    AUSAXS_CUDA(cudaMemsetAsync(cells.p, 0, align_up(ncells, 256) + 8, C.stream));
    hydration_add(C, cells.as<uint8_t>(), gmin, bins, atoms, ff, n, err);
    C.time_end(5, ev);
    generate(C, cells.as<uint8_t>(), gmin, bins, atoms, ff, n, noise, seed);
    int e = 0;
    AUSAXS_CUDA(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, C.stream));
    AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    if (e) throw Error{AUSAXS_ERR_ARGUMENT, "an atom lies outside the hydration grid"};
}

}  // namespace ausaxs_b200
