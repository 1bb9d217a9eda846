// Pair-distance histogram of points on the integer lattice by the autocorrelation of their occupancy.
//
// The grid model's excluded-volume dummies sit on a lattice of 1 A cells (RawGridExv places one per
// volume cell of the molecular grid, source/core/grid/exv/RawGridExv.cpp:10-59; at integer or at
// half-integer coordinates, depending on the grid's origin), and the reference bins their self pairs
// one by one (the exv-exv loop of HistogramManagerMTFFGrid.cpp:66-84).  Every pair's coordinate
// differences are then exact integers and its squared distance an integer s2 that the reference's
// float evaluation forms exactly (s2 < 2^24), so its bin and in-bin offset depend on s2 alone: the
// histogram is the sum over offsets (dx, dy, dz) of the number of point pairs with that offset, each
// offset binned once -- by the SIMD evaluators' rule; the few pairs of the scalar tail whose distance
// is an exact rounding tie are moved afterwards (lattice_tail_kernel).
//
// Counting the pairs per offset: the occupancy is stored as bit lines along x (one u32 word per 32
// cells).  For a line offset (dy, dz) a warp walks every pair of non-empty lines (y, z), (y + dy,
// z + dz) and lane l accumulates, for every x-shift s = 32 g + l, popc(P & (Q >> s)) (pairs with
// x2 - x1 = s) and popc(Q & (P >> s)) (x1 - x2 = s), with funnel shifts across words.  Every
// unordered pair appears once: each line offset is visited with dz > 0, or dz = 0 and dy > 0, or
// within a line (dy = dz = 0, s > 0 only).  Per line pair and lane this is words * (words + 1)
// AND + POPC terms against (points per line)^2 pair evaluations of the pair kernel, and the lines,
// the line table and a per-CTA histogram stay in shared memory.
//
// The counts and the fixed-point offset sums it produces are the integers the pair kernel adds for the
// same points, so the finalisation and everything after it see identical accumulators.
#include <algorithm>
#include <climits>
#include <cmath>

#include "lattice.cuh"

namespace ausaxs_b200 {

namespace {

__global__ void lattice_scan_init(int* st) {
    if (threadIdx.x == 0) {
        st[0] = st[1] = st[2] = INT_MAX;
        st[3] = st[4] = st[5] = INT_MIN;
        st[6] = 0;
        st[7] = 0;
    }
}

// Cell index of a lattice coordinate: floor(v) (v an integer or an integer + 1/2)
__device__ __forceinline__ int lattice_cell(float v) { return static_cast<int>(floorf(v)); }

// Every coordinate must be an integer, or an integer + 1/2, of magnitude below 2^20, with one kind
// per axis (st[7]: bit 2k integers seen on axis k, bit 2k + 1 half-integers): the difference of two
// such floats is then an exact integer.
__global__ void lattice_scan_kernel(const float4* p, int n, int* st) {
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    int bad = 0, kinds = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = p[i];
        const float c[3] = {v.x, v.y, v.z};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float t = 2.0f * c[k];  // exact below 2^20
            if (!(t == rintf(t) && fabsf(c[k]) < 1048576.0f)) {  // NaN fails the comparison
                bad = 1;
                continue;
            }
            kinds |= (c[k] == rintf(c[k]) ? 1 : 2) << (2 * k);
            const int iv = lattice_cell(c[k]);
            lo[k] = min(lo[k], iv);
            hi[k] = max(hi[k], iv);
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    for (int o = 16; o > 0; o >>= 1) kinds |= __shfl_xor_sync(0xffffffffu, kinds, o);
    bad = __any_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (lo[k] != INT_MAX) atomicMin(&st[k], lo[k]);
            if (hi[k] != INT_MIN) atomicMax(&st[3 + k], hi[k]);
        }
        if (bad) atomicOr(&st[6], 1);
        if (kinds) atomicOr(&st[7], kinds);
    }
}

struct BuildArgs {
    const float4* p;
    int n;
    int lo[3];
    int lx, ly, lz, words;
    uint32_t* grid;
    int* info;
};

__global__ void lattice_set_kernel(BuildArgs A) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const float4 v = A.p[i];
        const int x = lattice_cell(v.x) - A.lo[0];
        const int y = lattice_cell(v.y) - A.lo[1];
        const int z = lattice_cell(v.z) - A.lo[2];
        // every coordinate lies in [lo, hi] by the scan; checked once more before the write
        if (x < 0 || x >= A.lx || y < 0 || y >= A.ly || z < 0 || z >= A.lz) {
            atomicOr(&A.info[1], 2);
            continue;
        }
        const size_t w = (static_cast<size_t>(z) * A.ly + y) * A.words + (x >> 5);
        const uint32_t bit = 1u << (x & 31);
        if (atomicOr(&A.grid[w], bit) & bit) atomicOr(&A.info[1], 1);  // two points share a cell
    }
}

// one CTA of 1024 threads: non-empty lines in (z, y) order into the compact store, the table, the count
__global__ void __launch_bounds__(1024) lattice_compact_kernel(const uint32_t* grid, int n_lines_all, int words,
                                                               uint32_t* lines, int32_t* table, int* info) {
    __shared__ int warp_sum[32];
    __shared__ int s_base;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n_lines_all; base += 1024) {
        const int l = base + threadIdx.x;
        bool ne = false;
        if (l < n_lines_all)
            for (int w = 0; w < words; ++w) ne |= grid[static_cast<size_t>(l) * words + w] != 0u;
        const unsigned m = __ballot_sync(0xffffffffu, ne);
        if (lane == 0) warp_sum[warp] = __popc(m);
        __syncthreads();
        int before = 0;
        for (int k = 0; k < warp; ++k) before += warp_sum[k];
        const int pos = s_base + before + __popc(m & ((1u << lane) - 1u));
        if (l < n_lines_all) {
            table[l] = ne ? pos : -1;
            if (ne)
                for (int w = 0; w < words; ++w)
                    lines[static_cast<size_t>(pos) * words + w] = grid[static_cast<size_t>(l) * words + w];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int k = 0; k < 32; ++k) tot += warp_sum[k];
            s_base += tot;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) info[0] = s_base;
}

// threads per CTA: one CTA per SM holds the whole line store, so its warps are all the SM has
template <int W>
constexpr int lattice_threads() { return W <= 4 ? 1024 : kLatticeThreads; }

// Carry-save accumulation of popcounts (the Harley-Seal method) for x-shift group 0, the group with
// the most terms (2 W per line pair): the terms are added bitwise into words of weight 1 (ones) and
// 2 (twos) carried across line pairs, and only the words of weight 4 that fall out are popcounted.
// POPC issues on the XU pipe at a quarter of the ALU rate and binds the kernel; group 0 this way takes
// one POPC per four terms, the other groups keep one per term (carry-saving every group moves the
// bound onto the ALU pipe and is slower).  The count is 4 n + 2 popc(twos) + popc(ones).
struct CsaCount {
    uint32_t ones, twos, n;
};

// full adder over 32 bit positions: a + b + c = 2 hi + lo
__device__ __forceinline__ void csa(uint32_t& hi, uint32_t& lo, uint32_t a, uint32_t b, uint32_t c) {
    const uint32_t u = a ^ b;
    hi = (a & b) | (u & c);
    lo = u ^ c;
}

__device__ __forceinline__ void csa_add4(CsaCount& k, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    uint32_t t1, t2, f;
    csa(t1, k.ones, k.ones, a, b);
    csa(t2, k.ones, k.ones, c, d);
    csa(f, k.twos, k.twos, t1, t2);
    k.n += __popc(f);
}

__device__ __forceinline__ void csa_add2(CsaCount& k, uint32_t a, uint32_t b) {
    uint32_t t1;
    csa(t1, k.ones, k.ones, a, b);
    const uint32_t f = k.twos & t1;
    k.twos ^= t1;
    k.n += __popc(f);
}

__device__ __forceinline__ uint32_t csa_total(const CsaCount& k) {
    return 4u * k.n + 2u * static_cast<uint32_t>(__popc(k.twos)) + static_cast<uint32_t>(__popc(k.ones));
}

template <int W>
__global__ void __launch_bounds__(lattice_threads<W>(), 1) lattice_kernel(LatticeLaunch L) {
    constexpr int NTH = lattice_threads<W>();
    extern __shared__ __align__(16) unsigned char smem[];
    const int ly = L.G.ly, lz = L.G.lz, nb = L.nbins;
    uint32_t* s_lines = reinterpret_cast<uint32_t*>(smem);
    size_t off = (static_cast<size_t>(L.G.n_lines) * W * 4 + 15) & ~static_cast<size_t>(15);
    int32_t* s_table = reinterpret_cast<int32_t*>(smem + off);
    off += (static_cast<size_t>(ly) * lz * 4 + 15) & ~static_cast<size_t>(15);
    unsigned long long* h_cnt = reinterpret_cast<unsigned long long*>(smem + off);  // [nb + 1]: last = overflow
    unsigned long long* h_ds = h_cnt + (nb + 1);                                     // [nb + 1]
    // the grid's line store has exactly `words` words per line; W may round it up (3 -> 4)
    const int gw = L.G.words;
    for (int k = threadIdx.x; k < L.G.n_lines * W; k += NTH) {
        const int line = k / W, w = k - line * W;
        s_lines[k] = w < gw ? L.G.lines[static_cast<size_t>(line) * gw + w] : 0u;
    }
    for (int k = threadIdx.x; k < ly * lz; k += NTH) s_table[k] = L.G.table[k];
    for (int k = threadIdx.x; k < 2 * (nb + 1); k += NTH) h_cnt[k] = 0ull;
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int span = 2 * ly - 1;
    const float bin_limit = pair_bin_limit(nb);
    for (;;) {
        int item = 0;
        if (lane == 0) item = static_cast<int>(atomicAdd(L.counter, 1ull));
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= L.n_items) break;
        // item = (line offset, z chunk): the line offset's z1 range split into kLatticeChunks parts,
        // so the first (largest, dz = 0) offsets do not leave a long tail of lone warps
        const int base = item / kLatticeChunks;
        const int chunk = item - base * kLatticeChunks;
        const int dz = base / span;
        const int dy = base - dz * span - (ly - 1);
        if (dz == 0 && dy < 0) continue;  // the mirror image of an item with dy > 0
        const bool same = dz == 0 && dy == 0;
        uint32_t C[W];
#pragma unroll
        for (int g = 0; g < W; ++g) C[g] = 0u;
        const int y_lo = max(0, -dy), y_hi = min(ly, ly - dy);
        const int z_per = (lz - dz + kLatticeChunks - 1) / kLatticeChunks;
        const int z_begin = chunk * z_per, z_end = min(lz - dz, z_begin + z_per);
        if (!same) {
            // two lines: for x-shift group g, the terms P[w] & (Q >> s) and Q[w] & (P >> s) of every
            // word w, shift 32 g + lane; x-shift 0 (lane 0 of group 0) is counted once
            CsaCount K0{0u, 0u, 0u};
            const uint32_t not_lane0 = lane ? 0xffffffffu : 0u;
            for (int z1 = z_begin; z1 < z_end; ++z1) {
                const int32_t* t1 = s_table + z1 * ly;
                const int32_t* t2 = s_table + (z1 + dz) * ly + dy;
                for (int y1 = y_lo; y1 < y_hi; ++y1) {
                    const int i1 = t1[y1];
                    if (i1 < 0) continue;
                    const int i2 = t2[y1];
                    if (i2 < 0) continue;
                    uint32_t P[W], Q[W], Ps[W], Qs[W];
#pragma unroll
                    for (int w = 0; w < W; ++w) {
                        P[w] = s_lines[i1 * W + w];
                        Q[w] = s_lines[i2 * W + w];
                    }
#pragma unroll
                    for (int k = 0; k < W; ++k) {
                        Qs[k] = __funnelshift_r(Q[k], k + 1 < W ? Q[k + 1] : 0u, lane);
                        Ps[k] = __funnelshift_r(P[k], k + 1 < W ? P[k + 1] : 0u, lane);
                    }
#pragma unroll
                    for (int w = 0; w + 1 < W; w += 2)
                        csa_add4(K0, P[w] & Qs[w], Q[w] & Ps[w] & not_lane0, P[w + 1] & Qs[w + 1],
                                 Q[w + 1] & Ps[w + 1] & not_lane0);
                    if (W & 1) csa_add2(K0, P[W - 1] & Qs[W - 1], Q[W - 1] & Ps[W - 1] & not_lane0);
#pragma unroll
                    for (int g = 1; g < W; ++g) {
#pragma unroll
                        for (int w = 0; w + g < W; ++w)
                            C[g] += __popc(P[w] & Qs[w + g]) + __popc(Q[w] & Ps[w + g]);
                    }
                }
            }
            C[0] = csa_total(K0);
        } else {
            // a line with itself (one item per z range): the pairs x2 - x1 = s > 0 only
            for (int z1 = z_begin; z1 < z_end; ++z1) {
                const int32_t* t1 = s_table + z1 * ly;
                for (int y1 = 0; y1 < ly; ++y1) {
                    const int i1 = t1[y1];
                    if (i1 < 0) continue;
                    uint32_t P[W];
#pragma unroll
                    for (int w = 0; w < W; ++w) P[w] = s_lines[i1 * W + w];
#pragma unroll
                    for (int g = 0; g < W; ++g) {
#pragma unroll
                        for (int w = 0; w + g < W; ++w) {
                            const uint32_t pn = (w + g + 1 < W) ? P[w + g + 1] : 0u;
                            C[g] += __popc(P[w] & __funnelshift_r(P[w + g], pn, lane));
                        }
                    }
                }
            }
            if (lane == 0) C[0] = 0u;  // x-shift 0 within a line: a point with itself
        }
#pragma unroll
        for (int g = 0; g < W; ++g) {
            if (!C[g]) continue;
            const int s = 32 * g + lane;
            const int s2 = s * s + dy * dy + dz * dz;  // < 2^24: exact as a float
            // the reference's bin rule and the pair kernel's fixed-point in-bin offset (common.cuh)
            const float d = __fsqrt_rn(static_cast<float>(s2));
            const float xm = __fadd_rn(__fmul_rn(d, L.inv_w), kMagic);
            if (!(xm < bin_limit)) {
                atomicAdd(&h_cnt[nb], static_cast<unsigned long long>(C[g]));
                continue;
            }
            const int bin = __float_as_int(xm) - kMagicBits;
            atomicAdd(&h_cnt[bin], static_cast<unsigned long long>(C[g]));
            if (L.dsum) {
                const float r = __fmaf_rn(-__fsub_rn(xm, kMagic), L.c, d);
                const float t = __fmaf_rn(r, L.scale, kMagic);
                const unsigned long long res = static_cast<uint32_t>(__float_as_int(t) - kMagicBits + kResBias);
                atomicAdd(&h_ds[bin], res * C[g]);
            }
        }
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nb; b += NTH) {
        if (h_cnt[b]) atomicAdd(&L.counts[b], h_cnt[b]);
        if (L.dsum && h_ds[b]) atomicAdd(&L.dsum[b], h_ds[b]);
    }
    if (threadIdx.x == 0 && h_cnt[nb]) atomicAdd(L.overflow, h_cnt[nb]);
}

// The reference bins the last (row length mod 4) partners of every row with its scalar evaluator,
// which rounds ties away from zero (common.cuh::pair_eval); the lattice kernel used the SIMD rule (ties
// to even) for every pair.  For the self pairs i < j of n points, row i's scalar partners are
// j >= n - ((n - i - 1) & 3): at most 3 per row.  Where the two rules give different bins (an exact
// half-integer distance in bin units) the pair's count and offset move to the scalar rule's bin.
__global__ void lattice_tail_kernel(LatticeLaunch L) {
    const int n = L.n_pts;
    const float bin_limit = pair_bin_limit(L.nbins);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = L.pts[i];
        const int ts = n - ((n - i - 1) & 3);
        for (int j = ts > i + 1 ? ts : i + 1; j < n; ++j) {
            const float4 b = L.pts[j];
            const PairBin simd = pair_eval(a, b, L.inv_w, false);
            const PairBin tail = pair_eval(a, b, L.inv_w, true);
            if (simd.bin == tail.bin) continue;
            // the pair leaves the SIMD rule's bin (or the overflow count) for the scalar rule's
            const bool in0 = static_cast<unsigned>(simd.bin) < static_cast<unsigned>(L.nbins) &&
                             __fadd_rn(simd.xr, kMagic) < bin_limit;
            const bool in1 = static_cast<unsigned>(tail.bin) < static_cast<unsigned>(L.nbins);
            if (in0) {
                atomicAdd(&L.counts[simd.bin], ~0ull);  // -1 (two's complement: the total stays exact)
                if (L.dsum) atomicAdd(&L.dsum[simd.bin], 0ull - pair_residual(simd, L.c, L.scale));
            } else {
                atomicAdd(L.overflow, ~0ull);
            }
            if (in1) {
                atomicAdd(&L.counts[tail.bin], 1ull);
                if (L.dsum) atomicAdd(&L.dsum[tail.bin], static_cast<unsigned long long>(pair_residual(tail, L.c, L.scale)));
            } else {
                atomicAdd(L.overflow, 1ull);
            }
        }
    }
}

template <int W>
void launch_w(const LatticeLaunch& L, int grid, size_t smem, cudaStream_t s) {
    cudaFuncSetAttribute(lattice_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    lattice_kernel<W><<<grid, lattice_threads<W>(), smem, s>>>(L);
}

}  // namespace

void lattice_scan_launch(const float4* p, int n, int* stats, int sm_count, cudaStream_t s) {
    lattice_scan_init<<<1, 32, 0, s>>>(stats);
    const int grid = std::max(1, std::min(sm_count * 4, (n + 255) / 256));
    lattice_scan_kernel<<<grid, 256, 0, s>>>(p, n, stats);
}

void lattice_build_launch(const float4* p, int n, const int lo[3], int lx, int ly, int lz, int words, uint32_t* grid,
                          uint32_t* lines, int32_t* table, int* info, int sm_count, cudaStream_t s) {
    BuildArgs A{p, n, {lo[0], lo[1], lo[2]}, lx, ly, lz, words, grid, info};
    const int g = std::max(1, std::min(sm_count * 4, (n + 255) / 256));
    lattice_set_kernel<<<g, 256, 0, s>>>(A);
    lattice_compact_kernel<<<1, 1024, 0, s>>>(grid, ly * lz, words, lines, table, info);
}

bool lattice_rules_agree(long long s2_max, float inv_w) {
    // x = fl(fl(sqrt(s2)) * inv_w) exactly as the device and the reference's evaluators form it (IEEE
    // single precision, correctly rounded square root); the rules differ only when x is a half-integer
    for (long long s2 = 1; s2 <= s2_max; ++s2) {
        const float d = std::sqrt(static_cast<float>(s2));
        const float x = d * inv_w;
        if (x - std::floor(x) == 0.5f) return false;
    }
    return true;
}

void lattice_launch(const LatticeLaunch& L, int grid, size_t smem, cudaStream_t s) {
    switch (lattice_kernel_words(L.G.words)) {
        case 1: launch_w<1>(L, grid, smem, s); break;
        case 2: launch_w<2>(L, grid, smem, s); break;
        case 4: launch_w<4>(L, grid, smem, s); break;
        default: launch_w<8>(L, grid, smem, s); break;
    }
    if (L.tail_fix) {
        const int g = std::max(1, std::min(grid * 2, (L.n_pts + 255) / 256));
        lattice_tail_kernel<<<g, 256, 0, s>>>(L);
    }
}

}  // namespace ausaxs_b200
