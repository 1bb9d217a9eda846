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
constexpr int kScanBlock = 1024;  // cells per compaction block

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

// A_CENTER / W_CENTER for the cells holding atom / water centres, and the atoms' bin box (reduced per
// warp first; the loop runs warp-uniformly so every lane takes part in the reductions)
__global__ void mark_centres(const float4* __restrict__ atoms, int na, const float4* __restrict__ waters, int nw,
                             GridShape G, uint32_t* grid, int* box) {
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < na + nw; base += stride) {
        const int t = base + lane;
        const bool live = t < na + nw;
        const float4 p = !live ? make_float4(0.f, 0.f, 0.f, 0.f) : (t < na ? atoms[t] : waters[t - na]);
        const int i = to_bin(p.x, G.gmin[0]), j = to_bin(p.y, G.gmin[1]), k = to_bin(p.z, G.gmin[2]);
        if (base < na) {  // warp-uniform: this warp holds atoms
            const bool atom = t < na;
            const int lo[3] = {atom ? -i : INT_MIN, atom ? -j : INT_MIN, atom ? -k : INT_MIN};
            const int hi[3] = {atom ? i + 1 : INT_MIN, atom ? j + 1 : INT_MIN, atom ? k + 1 : INT_MIN};
            for (int d = 0; d < 3; ++d) {
                const int l = __reduce_max_sync(0xffffffffu, lo[d]);
                const int h = __reduce_max_sync(0xffffffffu, hi[d]);
                if (lane == 0) {
                    atomicMax(&box[d], l);
                    atomicMax(&box[3 + d], h);
                }
            }
        }
        if (!live || i < 0 || j < 0 || k < 0 || i >= G.bins[0] || j >= G.bins[1] || k >= G.bins[2]) continue;
        atomicOr(&grid[cell_index(G, i, j, k)], t < na ? kACenter : kWCenter);
    }
}

// One thread per (atom, x column, y column) of the atom's box bin +- ceil(r): the cells of that column
// within r = max(r_vdw, rvol) of the atom get kSphere (distances as the reference forms them:
// ((x - ax)^2 + (y - ay)^2) + (z - az)^2 in double).  Cells holding a water centre are masked when the
// grid is swept (kept()), so the OR needs no read of the cell first.
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

__device__ __forceinline__ bool kept(const GridShape& G, const Window& W, const uint32_t* grid, size_t L) {
    int i, j, k;
    cell_of(G, static_cast<uint32_t>(L), i, j, k);
    if (i < W.lo[0] || i >= W.hi[0] || j < W.lo[1] || j >= W.hi[1] || k < W.lo[2] || k >= W.hi[2]) return false;
    const uint32_t v = grid[L];
    return (v & kACenter) || ((v & kSphere) && !(v & kWCenter));
}

__global__ void count_kept(GridShape G, const int* box, const uint32_t* grid, size_t cells, unsigned int* block_counts) {
    __shared__ unsigned int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const Window W = window(G, box);
    const size_t L = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x;
    const bool k = L < cells && kept(G, W, grid, L);
    const unsigned int warp_n = __popc(__ballot_sync(0xffffffffu, k));
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

__global__ void write_kept(GridShape G, const int* box, const uint32_t* grid, size_t cells, const unsigned int* offsets,
                           float4* out, long long cap) {
    __shared__ unsigned int warp_base[kScanBlock / 32];
    const Window W = window(G, box);
    const size_t L = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x;
    const bool k = L < cells && kept(G, W, grid, L);
    const unsigned int mask = __ballot_sync(0xffffffffu, k);
    if ((threadIdx.x & 31) == 0) warp_base[threadIdx.x >> 5] = __popc(mask);
    __syncthreads();
    if (threadIdx.x == 0) {  // exclusive prefix over the block's warps, in order
        unsigned int acc = 0;
        for (int w = 0; w < kScanBlock / 32; ++w) {
            const unsigned int c = warp_base[w];
            warp_base[w] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (!k) return;
    const unsigned int lane_rank = __popc(mask & ((1u << (threadIdx.x & 31)) - 1u));
    const long long pos = static_cast<long long>(offsets[blockIdx.x]) + warp_base[threadIdx.x >> 5] + lane_rank;
    if (pos >= cap) return;
    int ii, jj, kk;
    cell_of(G, static_cast<uint32_t>(L), ii, jj, kk);
    out[pos] = make_float4(static_cast<float>(G.gmin[0] + ii), static_cast<float>(G.gmin[1] + jj),
                           static_cast<float>(G.gmin[2] + kk), __int_as_float(0));  // form_factor_t EXCLUDED_VOLUME
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
    if (cells >= (size_t)1 << 32) throw Error{AUSAXS_ERR_CAPACITY, "excluded-volume grid of 2^32 cells or more"};
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
    count_kept<<<(unsigned)nblocks, kScanBlock, 0, s>>>(G, box, grid, cells, counts);
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
    write_kept<<<(unsigned)nblocks, kScanBlock, 0, s>>>(G, box, grid, cells, counts, dst, (long long)n);
    C.check_launch("grid write");
    C.time_end(4, ev);
}

}  // namespace ausaxs_b200
