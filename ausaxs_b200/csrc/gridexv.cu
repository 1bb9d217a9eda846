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
    int win_lo[3], win_hi[3];  // sweep window (cells), half-open
};

__device__ __forceinline__ size_t cell_index(const GridShape& G, int i, int j, int k) {
    return (static_cast<size_t>(i) * G.bins[1] + j) * G.bins[2] + k;
}

__device__ __forceinline__ int to_bin(double v, double lo) { return static_cast<int>(round(v - lo)); }

__global__ void mark_centres(const float4* __restrict__ atoms, int na, const float4* __restrict__ waters, int nw,
                             GridShape G, uint32_t* grid) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + nw; t += gridDim.x * blockDim.x) {
        const float4 p = t < na ? atoms[t] : waters[t - na];
        const int i = to_bin(p.x, G.gmin[0]), j = to_bin(p.y, G.gmin[1]), k = to_bin(p.z, G.gmin[2]);
        if (i < 0 || j < 0 || k < 0 || i >= G.bins[0] || j >= G.bins[1] || k >= G.bins[2]) continue;
        atomicOr(&grid[cell_index(G, i, j, k)], t < na ? kACenter : kWCenter);
    }
}

// one thread per atom: the cells of its box bin +- ceil(r) within r = max(r_vdw, rvol) of the atom
// (distances as the reference forms them: ((x - ax)^2 + (y - ay)^2) + (z - az)^2 in double)
__global__ void mark_spheres(const float4* __restrict__ atoms, int na, GridShape G, uint32_t* grid) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const float4 p = atoms[a];
        const int ff = __float_as_int(p.w);
        const double rv = (ff >= 0 && ff < kNff) ? c_vdw[ff] : 0.0;
        const double rvdw2 = rv * rv, rvol2 = kRvol * kRvol;
        const double r = fmax(rv, kRvol);
        const int br = static_cast<int>(ceil(r));
        const double ax = p.x, ay = p.y, az = p.z;
        const int bx = to_bin(ax, G.gmin[0]), by = to_bin(ay, G.gmin[1]), bz = to_bin(az, G.gmin[2]);
        const int i0 = max(bx - br, 0), i1 = min(bx + br + 1, G.bins[0]);
        const int j0 = max(by - br, 0), j1 = min(by + br + 1, G.bins[1]);
        const int k0 = max(bz - br, 0), k1 = min(bz + br + 1, G.bins[2]);
        for (int i = i0; i < i1; ++i) {
            // no contraction: every product and sum rounded on its own, as the restated loop forms them
            const double dx = __dsub_rn(__dadd_rn(G.gmin[0], (double)i), ax);
            const double x2 = __dmul_rn(dx, dx);
            for (int j = j0; j < j1; ++j) {
                const double dy = __dsub_rn(__dadd_rn(G.gmin[1], (double)j), ay);
                const double x2y2 = __dadd_rn(x2, __dmul_rn(dy, dy));
                for (int k = k0; k < k1; ++k) {
                    const double dz = __dsub_rn(__dadd_rn(G.gmin[2], (double)k), az);
                    const double dist = __dadd_rn(x2y2, __dmul_rn(dz, dz));
                    if (dist <= rvdw2 || dist <= rvol2) {
                        uint32_t* c = &grid[cell_index(G, i, j, k)];
                        if (!(*c & kWCenter)) atomicOr(c, kSphere);  // water centres are marked before this pass
                    }
                }
            }
        }
    }
}

__device__ __forceinline__ bool kept(const GridShape& G, const uint32_t* grid, size_t L) {
    const int k = static_cast<int>(L % G.bins[2]);
    const int j = static_cast<int>((L / G.bins[2]) % G.bins[1]);
    const int i = static_cast<int>(L / (static_cast<size_t>(G.bins[2]) * G.bins[1]));
    if (i < G.win_lo[0] || i >= G.win_hi[0] || j < G.win_lo[1] || j >= G.win_hi[1] || k < G.win_lo[2] ||
        k >= G.win_hi[2])
        return false;
    const uint32_t v = grid[L];
    return (v & kACenter) || ((v & kSphere) && !(v & kWCenter));
}

__global__ void count_kept(GridShape G, const uint32_t* grid, size_t cells, unsigned int* block_counts) {
    __shared__ unsigned int s;
    if (threadIdx.x == 0) s = 0;
    __syncthreads();
    const size_t L = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x;
    const bool k = L < cells && kept(G, grid, L);
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

__global__ void write_kept(GridShape G, const uint32_t* grid, size_t cells, const unsigned int* offsets, float4* out,
                           long long cap) {
    __shared__ unsigned int warp_base[kScanBlock / 32];
    const size_t L = static_cast<size_t>(blockIdx.x) * kScanBlock + threadIdx.x;
    const bool k = L < cells && kept(G, grid, L);
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
    const int kk = static_cast<int>(L % G.bins[2]);
    const int jj = static_cast<int>((L / G.bins[2]) % G.bins[1]);
    const int ii = static_cast<int>(L / (static_cast<size_t>(G.bins[2]) * G.bins[1]));
    out[pos] = make_float4(static_cast<float>(G.gmin[0] + ii), static_cast<float>(G.gmin[1] + jj),
                           static_cast<float>(G.gmin[2] + kk), __int_as_float(0));  // form_factor_t EXCLUDED_VOLUME
}

__global__ void atom_bin_box(const float4* __restrict__ atoms, int na, GridShape G, int* box) {
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
        const float4 p = atoms[a];
        const int b[3] = {to_bin(p.x, G.gmin[0]), to_bin(p.y, G.gmin[1]), to_bin(p.z, G.gmin[2])};
        for (int d = 0; d < 3; ++d) {
            atomicMin(&box[d], b[d]);
            atomicMax(&box[3 + d], b[d] + 1);
        }
    }
}

}  // namespace

void GridExv::run(Ctx& C, const float4* atoms, int na, const float4* waters, int nw, const float lo[3],
                  const float hi[3], bool want_points) {
    cudaStream_t s = C.stream;
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
    if (cells > (size_t)1 << 32) throw Error{AUSAXS_ERR_CAPACITY, "excluded-volume grid above 2^32 cells"};
    const size_t nblocks = (cells + kScanBlock - 1) / kScanBlock;
    const size_t grid_bytes = align_up(cells * 4, 256), cnt_bytes = align_up(nblocks * 4, 256);
    work.ensure(grid_bytes + cnt_bytes + 256);
    uint32_t* grid = work.as<uint32_t>();
    unsigned int* counts = work.as<unsigned int>(grid_bytes);
    unsigned long long* total = work.as<unsigned long long>(grid_bytes + cnt_bytes);
    int* box = reinterpret_cast<int*>(total + 1);
    AUSAXS_CUDA(cudaMemsetAsync(grid, 0, cells * 4, s));
    const int hbox[6] = {1 << 30, 1 << 30, 1 << 30, -(1 << 30), -(1 << 30), -(1 << 30)};
    AUSAXS_CUDA(cudaMemcpyAsync(box, hbox, sizeof(hbox), cudaMemcpyHostToDevice, s));  // pageable: staged on return
    const int threads = 256;
    const int blocks_pts = std::max(1, std::min((na + nw + threads - 1) / threads, C.sm_count * 8));
    mark_centres<<<blocks_pts, threads, 0, s>>>(atoms, na, waters, nw, G, grid);
    C.check_launch("grid centres");
    if (na > 0) {
        const int blocks_a = std::max(1, std::min((na + threads - 1) / threads, C.sm_count * 8));
        mark_spheres<<<blocks_a, threads, 0, s>>>(atoms, na, G, grid);
        C.check_launch("grid spheres");
        atom_bin_box<<<blocks_a, threads, 0, s>>>(atoms, na, G, box);
        C.check_launch("grid box");
    }
    int hb[6] = {0, 0, 0, 0, 0, 0};
    AUSAXS_CUDA(cudaMemcpyAsync(hb, box, sizeof(hb), cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    // sweep window (RawGridExv.cpp:35-41): the atoms' bin box widened by round(max(rvol, 2)) cells
    const int buffer = (int)std::max(1.0, std::round(std::max(kRvol, 2.0)));
    for (int d = 0; d < 3; ++d) {
        G.win_lo[d] = na > 0 ? std::max(hb[d] - buffer, 0) : 0;
        G.win_hi[d] = na > 0 ? std::min(hb[3 + d] + buffer + 1, G.bins[d]) : 0;
    }
    count_kept<<<(unsigned)nblocks, kScanBlock, 0, s>>>(G, grid, cells, counts);
    C.check_launch("grid count");
    scan_counts<<<1, 1024, 0, s>>>(counts, (int)nblocks, total);
    C.check_launch("grid scan");
    unsigned long long n = 0;
    AUSAXS_CUDA(cudaMemcpyAsync(&n, total, 8, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    count = (long long)n;
    volume = (double)n;  // cells of 1 A^3
    if (!want_points || n == 0) return;
    points.ensure(align_up(n * 16, 256));
    write_kept<<<(unsigned)nblocks, kScanBlock, 0, s>>>(G, grid, cells, counts, points.as<float4>(), (long long)n);
    C.check_launch("grid write");
}

}  // namespace ausaxs_b200

using namespace ausaxs_b200;

extern "C" int ausaxs_gpu_grid_exv(ausaxs_gpu_ctx* ctx, const float* atoms, int32_t n_atoms, const float* waters,
                                   int32_t n_waters, float* exv_out, int64_t capacity, int64_t* n_exv, double* volume) {
    return guarded([&] {
        if (!ctx || !n_exv || n_atoms < 0 || n_waters < 0 || (n_atoms && !atoms) || (n_waters && !waters) ||
            (capacity > 0 && !exv_out))
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        Structure S;  // census and validation of the points (form-factor types, finite coordinates)
        S.ctx = &C;
        S.load(atoms, n_atoms, waters, n_waters, nullptr, 0, 1, true);
        GridExv g;
        g.run(C, S.raw_a.as<float4>(), n_atoms, S.raw_w.as<float4>(), n_waters, S.lo, S.hi, capacity > 0);
        *n_exv = g.count;
        if (volume) *volume = g.volume;
        if (capacity > 0 && g.count > 0) {
            if (capacity < g.count) throw Error{AUSAXS_ERR_CAPACITY, "exv_out holds fewer records than the grid has dummies"};
            AUSAXS_CUDA(cudaMemcpyAsync(exv_out, g.points.p, (size_t)g.count * 16, cudaMemcpyDeviceToHost, C.stream));
            AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
        }
    });
}
