// Grid excluded-volume dummies on the device: what RawGridExv::create (source/core/grid/exv/RawGridExv.cpp:10-59)
// returns for the expanded molecular grid that HistogramManagerMTFFGrid::calculate_all() uses, and the
// grid volume that Molecule::get_volume_grid() returns (Grid.cpp:428-431), with the reference's default
// grid settings (cell width 1 A, rvol 2.15 A, exv width 1 A, AtomicOnly expansion).
//
// The reference marks cells one atom after another (SphericalExpander.h:27-76): A_CENTER / W_CENTER for
// the cells holding atom / water centres, then A_AREA for cells within an atom's van der Waals radius that
// hold nothing but VOLUME, and VOLUME for empty cells within (r_vdw, rvol].  The set of cells it finally
// keeps (A_CENTER, A_AREA or VOLUME) does not depend on that order: a cell is kept when it holds an atom
// centre, or when it holds no water centre and lies within max(r_vdw, rvol) of some atom.  So here every
// atom marks its sphere with atomic ORs in parallel, and the kept cells are compacted in the reference's
// sweep order (x, then y, then z) by a block-count / scan / write pass.
#include <algorithm>
#include <climits>
#include <cmath>

#include "engine.cuh"
#include "guard.cuh"
#include "gridexv.cuh"

namespace ausaxs_b200 {
namespace {

constexpr uint32_t kACenter = 1, kWCenter = 2, kSphere = 4;
constexpr double kRvol = 2.15;   // settings::grid::min_exv_radius (GridSettings.cpp:14)
constexpr int kScanThreads = 1024;                     // threads of a compaction block
constexpr int kCellsPerThread = 4;                     // consecutive cells per thread (one 16-byte load)
constexpr int kScanBlock = kScanThreads * kCellsPerThread;  // cells per compaction block

// constants::radius::get_vdw_radius(form_factor_t) (include/core/form_factor/FormFactorType.h:173-192):
// H 1.1, C-family 1.96, N-family 1.79, O / OH 1.71, S / SH 2.06, OTHER (Ar) 1.88 A
__constant__ double c_vdw[kNff] = {0.0, 1.71, 1.1, 1.96, 1.96, 1.96, 1.96, 1.79, 1.79, 1.79, 1.79, 1.71, 2.06, 2.06, 1.88};

struct GridShape {
    double gmin[3];
    int bins[3];
    int buffer;  // sweep window margin (cells) around the atoms' bin box
};

// The atoms' bin box, reduced with atomicMax only: box[d] = -min bin, box[3 + d] = max bin + 1.  A byte
// fill of 0x80 starts every word at -2139062144, below any bin, so no host-side initialisation is needed.
constexpr int kBoxFill = 0x80;

__device__ __forceinline__ size_t cell_index(const GridShape& G, int i, int j, int k) {
    return (static_cast<size_t>(i) * G.bins[1] + j) * G.bins[2] + k;
}

__device__ __forceinline__ int to_bin(double v, double lo) { return static_cast<int>(round(v - lo)); }

// A_CENTER / W_CENTER for the cells holding atom / water centres, and the atoms' bin box (reduced in
// registers, then per warp, then per block: one atomic per block and box word)
__global__ void mark_centres(const float4* __restrict__ atoms, int na, const float4* __restrict__ waters, int nw,
                             GridShape G, uint32_t* grid, int* box) {
    __shared__ int s_box[6];
    if (threadIdx.x < 6) s_box[threadIdx.x] = INT_MIN;
    __syncthreads();
    int r[6] = {INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN, INT_MIN};  // -min bin, max bin + 1
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + nw; t += gridDim.x * blockDim.x) {
        const float4 p = t < na ? atoms[t] : waters[t - na];
        const int i = to_bin(p.x, G.gmin[0]), j = to_bin(p.y, G.gmin[1]), k = to_bin(p.z, G.gmin[2]);
        if (t < na) {
            r[0] = max(r[0], -i), r[1] = max(r[1], -j), r[2] = max(r[2], -k);
            r[3] = max(r[3], i + 1), r[4] = max(r[4], j + 1), r[5] = max(r[5], k + 1);
        }
        if (i < 0 || j < 0 || k < 0 || i >= G.bins[0] || j >= G.bins[1] || k >= G.bins[2]) continue;
        atomicOr(&grid[cell_index(G, i, j, k)], t < na ? kACenter : kWCenter);
    }
#pragma unroll
    for (int d = 0; d < 6; ++d) {
        const int v = __reduce_max_sync(0xffffffffu, r[d]);
        if ((threadIdx.x & 31) == 0 && v != INT_MIN) atomicMax(&s_box[d], v);
    }
    __syncthreads();
    if (threadIdx.x < 6 && s_box[threadIdx.x] != INT_MIN) atomicMax(&box[threadIdx.x], s_box[threadIdx.x]);
}

// One thread per (atom, x column, y column) of the atom's box bin +- ceil(r): the cells of that column
// within r = max(r_vdw, rvol) of the atom get kSphere (distances as the reference forms them:
// ((x - ax)^2 + (y - ay)^2) + (z - az)^2 in double).  Cells holding a water centre are masked when the
// grid is swept (kept_bits), so the OR needs no read of the cell first.
constexpr int kSpan = 7;  // 2 * ceil(max r) + 1 cells: r <= 2.15 A for every form-factor type

__global__ void mark_spheres(const float4* __restrict__ atoms, int na, GridShape G, uint32_t* grid) {
    const long long total = static_cast<long long>(na) * kSpan * kSpan;
    for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
         t += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int a = static_cast<int>(t / (kSpan * kSpan));
        const int col = static_cast<int>(t - static_cast<long long>(a) * kSpan * kSpan);
        const float4 p = atoms[a];
        const int ff = __float_as_int(p.w);
        const double rv = (ff >= 0 && ff < kNff) ? c_vdw[ff] : 0.0;
        const double rvdw2 = rv * rv, rvol2 = kRvol * kRvol;
        const int br = static_cast<int>(ceil(fmax(rv, kRvol)));
        const int di = col / kSpan - kSpan / 2, dj = col % kSpan - kSpan / 2;
        if (di < -br || di > br || dj < -br || dj > br) continue;
        const double ax = p.x, ay = p.y, az = p.z;
        const int i = to_bin(ax, G.gmin[0]) + di, j = to_bin(ay, G.gmin[1]) + dj, bz = to_bin(az, G.gmin[2]);
        if (i < 0 || i >= G.bins[0] || j < 0 || j >= G.bins[1]) continue;
        const int k0 = max(bz - br, 0), k1 = min(bz + br + 1, G.bins[2]);
        // no contraction: every product and sum rounded on its own, as the restated loop forms them
        const double dx = __dsub_rn(__dadd_rn(G.gmin[0], (double)i), ax);
        const double dy = __dsub_rn(__dadd_rn(G.gmin[1], (double)j), ay);
        const double x2y2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
        uint32_t* column = grid + (static_cast<size_t>(i) * G.bins[1] + j) * G.bins[2];
        for (int k = k0; k < k1; ++k) {
            const double dz = __dsub_rn(__dadd_rn(G.gmin[2], (double)k), az);
            const double dist = __dadd_rn(x2y2, __dmul_rn(dz, dz));
            if (dist <= rvdw2 || dist <= rvol2) atomicOr(column + k, kSphere);
        }
    }
}

// sweep window (RawGridExv.cpp:35-41): the atoms' bin box widened by `buffer` cells, clipped to the grid;
// empty when there are no atoms (the box words keep their fill)
struct Window {
    int lo[3], hi[3];
};

__device__ __forceinline__ Window window(const GridShape& G, const int* box) {
    Window w;
    for (int d = 0; d < 3; ++d) {
        w.lo[d] = max(-box[d] - G.buffer, 0);
        w.hi[d] = min(box[3 + d] + G.buffer + 1, G.bins[d]);
    }
    return w;
}

// cell coordinates of linear index L (the grid holds fewer than 2^32 cells)
__device__ __forceinline__ void cell_of(const GridShape& G, uint32_t L, int& i, int& j, int& k) {
    const uint32_t row = L / static_cast<uint32_t>(G.bins[2]);
    k = static_cast<int>(L - row * static_cast<uint32_t>(G.bins[2]));
    i = static_cast<int>(row / static_cast<uint32_t>(G.bins[1]));
    j = static_cast<int>(row - static_cast<uint32_t>(i) * static_cast<uint32_t>(G.bins[1]));
}

// The kept flags of the kCellsPerThread consecutive cells starting at L (bit c: cell L + c), in sweep
// order; cells at or beyond `cells` are not kept.  One index decomposition per thread, the following
// cells step k with carries into j and i.
__device__ __forceinline__ uint32_t kept_bits(const GridShape& G, const Window& W, const uint32_t* grid, uint32_t L,
                                              uint32_t cells) {
    if (L >= cells) return 0u;
    uint32_t v[kCellsPerThread];
    if (L + kCellsPerThread <= cells) {
        const uint4 q = *reinterpret_cast<const uint4*>(grid + L);  // L is a multiple of 4: 16-byte aligned
        v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
    } else {
#pragma unroll
        for (int c = 0; c < kCellsPerThread; ++c) v[c] = L + c < cells ? grid[L + c] : 0u;
    }
    int i, j, k;
    cell_of(G, L, i, j, k);
    uint32_t bits = 0;
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) {
        const bool in = i >= W.lo[0] && i < W.hi[0] && j >= W.lo[1] && j < W.hi[1] && k >= W.lo[2] && k < W.hi[2];
        const bool keep = (v[c] & kACenter) || ((v[c] & kSphere) && !(v[c] & kWCenter));
        if (in && keep && L + c < cells) bits |= 1u << c;
        if (++k == G.bins[2]) {
            k = 0;
            if (++j == G.bins[1]) j = 0, ++i;
        }
    }
    return bits;
}

__global__ void count_kept(GridShape G, const int* box, const uint32_t* grid, uint32_t cells, unsigned int* block_counts) {
    __shared__ unsigned int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const Window W = window(G, box);
    const uint32_t L = blockIdx.x * kScanBlock + threadIdx.x * kCellsPerThread;
    const unsigned int warp_n = __reduce_add_sync(0xffffffffu, __popc(kept_bits(G, W, grid, L, cells)));
    if ((threadIdx.x & 31) == 0 && warp_n) atomicAdd(&s, warp_n);
    __syncthreads();
    if (threadIdx.x == 0) block_counts[blockIdx.x] = s;
}

// exclusive scan of the block counts (one block; the counts fit in shared memory passes)
__global__ void scan_counts(unsigned int* counts, int n, unsigned long long* total) {
    __shared__ unsigned long long carry;
    __shared__ unsigned int warp_sums[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const unsigned int v = t < n ? counts[t] : 0u;
        // inclusive warp scan
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
            if (threadIdx.x < nw) warp_sums[threadIdx.x] = w;  // inclusive over warps
        }
        __syncthreads();
        const unsigned int warp_prefix = (threadIdx.x >> 5) ? warp_sums[(threadIdx.x >> 5) - 1] : 0u;
        const unsigned long long excl = carry + warp_prefix + x - v;
        const unsigned int block_total = warp_sums[(blockDim.x >> 5) - 1];
        __syncthreads();
        if (t < n) counts[t] = static_cast<unsigned int>(excl);
        if (threadIdx.x == 0) carry += block_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void write_kept(GridShape G, const int* box, const uint32_t* grid, uint32_t cells, const unsigned int* offsets,
                           float4* out, long long cap) {
    constexpr int kWarps = kScanThreads / 32;
    __shared__ unsigned int warp_base[kWarps];
    const Window W = window(G, box);
    const uint32_t L = blockIdx.x * kScanBlock + threadIdx.x * kCellsPerThread;
    const uint32_t bits = kept_bits(G, W, grid, L, cells);
    const int lane = threadIdx.x & 31;
    // inclusive scan of the per-thread counts within the warp, then the warps' bases in order
    const unsigned int n = __popc(bits);
    unsigned int x = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_base[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int acc = 0;
        for (int w = 0; w < kWarps; ++w) {
            const unsigned int c = warp_base[w];
            warp_base[w] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (!bits) return;
    long long pos = static_cast<long long>(offsets[blockIdx.x]) + warp_base[threadIdx.x >> 5] + (x - n);
    int i, j, k;
    cell_of(G, L, i, j, k);
#pragma unroll
    for (int c = 0; c < kCellsPerThread; ++c) {
        if (bits & (1u << c)) {
            if (pos < cap)
                out[pos] = make_float4(static_cast<float>(G.gmin[0] + i), static_cast<float>(G.gmin[1] + j),
                                       static_cast<float>(G.gmin[2] + k), __int_as_float(0));  // EXCLUDED_VOLUME
            ++pos;
        }
        if (++k == G.bins[2]) {
            k = 0;
            if (++j == G.bins[1]) j = 0, ++i;
        }
    }
}

}  // namespace

void GridExv::run(Ctx& C, const float4* atoms, int na, const float4* waters, int nw, const float lo[3],
                  const float hi[3], bool want_points, float4* out, long long cap) {
    cudaStream_t s = C.stream;
    count = 0;
    volume = 0;
    // axes (Grid.cpp:34-102): bounding box of atoms, waters and the origin
    double mn[3], mx[3];
    for (int d = 0; d < 3; ++d) {
        mn[d] = std::min(0.0, (double)lo[d]);
        mx[d] = std::max(0.0, (double)hi[d]);
    }
    const double diff[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    const double scaling = (diff[0] < 50 || diff[1] < 50 || diff[2] < 50) ? 1.0 : 0.25;
    const double margin = 2.14 + 1.71 + (-0.35) + 3.0;  // r_vdw(P) + r_vdw(O) + shell correction + 3 cells
    GridShape G{};
    size_t cells = 1;
    for (int d = 0; d < 3; ++d) {
        const double e = std::max(0.5 * diff[d] * scaling, margin);
        G.gmin[d] = std::floor(mn[d] - e - 1.0);
        const double gmax = std::ceil(mx[d] + e + 1.0);
        G.bins[d] = (int)(gmax - G.gmin[d]);
        cells *= (size_t)G.bins[d];
    }
    // 32-bit cell indices, with room for the last compaction block's overhang
    if (cells >= ((size_t)1 << 32) - kScanBlock) throw Error{AUSAXS_ERR_CAPACITY, "excluded-volume grid of 2^32 cells or more"};
    G.buffer = (int)std::max(1.0, std::round(std::max(kRvol, 2.0)));  // round(max(rvol, 2)) cells
    const size_t nblocks = (cells + kScanBlock - 1) / kScanBlock;
    const size_t grid_bytes = align_up(cells * 4, 256), cnt_bytes = align_up(nblocks * 4, 256);
    work.ensure(grid_bytes + cnt_bytes + 256);
    uint32_t* grid = work.as<uint32_t>();
    unsigned int* counts = work.as<unsigned int>(grid_bytes);
    unsigned long long* total = work.as<unsigned long long>(grid_bytes + cnt_bytes);
    int* box = reinterpret_cast<int*>(total + 1);
    cudaEvent_t ev;
    C.time_begin(4, &ev);
    AUSAXS_CUDA(cudaMemsetAsync(grid, 0, cells * 4, s));
    AUSAXS_CUDA(cudaMemsetAsync(box, kBoxFill, 6 * sizeof(int), s));
    const int threads = 256;
    const int blocks_pts = std::max(1, std::min((na + nw + threads - 1) / threads, C.sm_count * 8));
    mark_centres<<<blocks_pts, threads, 0, s>>>(atoms, na, waters, nw, G, grid, box);
    C.check_launch("grid centres");
    if (na > 0) {
        const long long columns = (long long)na * kSpan * kSpan;
        const int blocks_s = (int)std::max(1LL, std::min((columns + threads - 1) / threads, (long long)C.sm_count * 16));
        mark_spheres<<<blocks_s, threads, 0, s>>>(atoms, na, G, grid);
        C.check_launch("grid spheres");
    }
    count_kept<<<(unsigned)nblocks, kScanThreads, 0, s>>>(G, box, grid, (uint32_t)cells, counts);
    C.check_launch("grid count");
    scan_counts<<<1, 1024, 0, s>>>(counts, (int)nblocks, total);
    C.check_launch("grid scan");
    C.time_end(4, ev);
    unsigned long long n = 0;  // the one synchronisation: the dummy count sizes the output
    AUSAXS_CUDA(cudaMemcpyAsync(&n, total, 8, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    count = (long long)n;
    volume = (double)n;  // cells of 1 A^3
    if (!want_points || n == 0) return;
    float4* dst = out;
    if (!dst) {
        points.ensure(align_up(n * 16, 256));
        dst = points.as<float4>();
    } else if (cap < (long long)n) {
        throw Error{AUSAXS_ERR_CAPACITY, "exv_out holds fewer records than the grid has dummies"};
    }
    C.time_begin(4, &ev);
    write_kept<<<(unsigned)nblocks, kScanThreads, 0, s>>>(G, box, grid, (uint32_t)cells, counts, dst, (long long)n);
    C.check_launch("grid write");
    C.time_end(4, ev);
}

}  // namespace ausaxs_b200
