// Split-BF16 tensor-core contraction of the Debye transform (the K4 stage) on sm_100a.
//
//   sinqd[r][q] = sum_b H[r][b] * sinc(q * d_g(r)[b])
//
// is the dense product of the histogram rows H [R x B] with the sinc table S [B x Q]
// (CompositeDistanceHistogramFFAvgBase.cpp:427-467 computes it as R*Q inner products in FP64).
// Each CTA owns a 128-row x 128-q tile of one K split (a contiguous bin range) for one distance
// axis g; the partial sums of the splits are added in FP64 by the epilogue (debye.cu).
//   * staging: threads m and m + 128 convert row m of H (FP64 -> FP32) for the chunk's 64 bins and splits it
//     into three BF16 terms hi + mid + lo (exact for an FP32 value); thread n generates the sinc
//     values of q n on the fly from the distance axis (FP32) and splits them likewise; rounded-up
//     BF16 magnitudes |H|, |S| go to two more tiles.  Tiles use the no-swizzle K-major core-matrix
//     layout (8 rows x 16 bytes), written as 16-byte vectors;
//   * one elected thread issues tcgen05.mma kind::f16 (BF16 x BF16 -> FP32): hi*hi into the main
//     accumulator, hi*mid + mid*hi + hi*lo + lo*hi + mid*mid into a correction accumulator (kept
//     apart so the small terms do not add rounding to the large sum), |H|*|S| into a bound
//     accumulator, then tcgen05.commit to an mbarrier;
//   * after the last chunk every warp reads its 32 TMEM lanes (tcgen05.ld) and stores
//     main + correction and the bound in FP32; the CTAs of the first q tile also store sum_b |H|.
// Every wait is bounded: on timeout the kernel records an error flag, waits (bounded) for its MMAs,
// frees its tensor memory and returns; the epilogue then uses FP64 for every q.
#include <algorithm>

#include "debye.cuh"

namespace ausaxs_b200 {
namespace {

constexpr int kM = 128;         // rows per CTA (UMMA M)
constexpr int kN = 128;         // q values per CTA (UMMA N)
constexpr int kKC = 64;         // bins per staged chunk (4 UMMA K-steps of 16)
constexpr int kThreadsTC = 256;  // two threads per operand row / q column (halves of a K chunk)
constexpr int kTileBytes = kM * kKC * 2;  // one BF16 operand tile, 16 KiB
constexpr int kTmemCols = 512;            // main, correction, bound accumulators (128 columns each)
constexpr int kColCorr = kN, kColBound = 2 * kN;
constexpr long long kSpinLimit = 1ll << 22;

__device__ __forceinline__ unsigned short bf16_rn(float x) {
    // round-to-nearest-even FP32 -> BF16 (finite inputs)
    unsigned int u = __float_as_uint(x);
    u += 0x7fffu + ((u >> 16) & 1u);
    return static_cast<unsigned short>(u >> 16);
}
__device__ __forceinline__ unsigned short bf16_mag_up(float x) {
    // |x| rounded up to BF16 (finite inputs): an upper bound of the magnitude
    unsigned int u = __float_as_uint(x) & 0x7fffffffu;
    if (u & 0xffffu) u += 0x10000u;
    return static_cast<unsigned short>(u >> 16);
}
__device__ __forceinline__ float bf16_to_f(unsigned short h) { return __uint_as_float(static_cast<unsigned int>(h) << 16); }

// Splits eight FP32 values into the four BF16 operand vectors (8 elements = 16 bytes each).
struct Split8 {
    uint4 hi, mid, lo, mag;
};
__device__ __forceinline__ Split8 split8(const float (&v)[8]) {
    uint32_t h[4], m[4], l[4], a[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        uint32_t hh[2], mm[2], ll[2], aa[2];
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const float x = v[2 * j + t];
            const unsigned short xh = bf16_rn(x);
            const float r1 = x - bf16_to_f(xh);
            const unsigned short xm = bf16_rn(r1);
            hh[t] = xh;
            mm[t] = xm;
            ll[t] = bf16_rn(r1 - bf16_to_f(xm));
            aa[t] = bf16_mag_up(x);
        }
        h[j] = hh[0] | (hh[1] << 16);
        m[j] = mm[0] | (mm[1] << 16);
        l[j] = ll[0] | (ll[1] << 16);
        a[j] = aa[0] | (aa[1] << 16);
    }
    return Split8{make_uint4(h[0], h[1], h[2], h[3]), make_uint4(m[0], m[1], m[2], m[3]),
                  make_uint4(l[0], l[1], l[2], l[3]), make_uint4(a[0], a[1], a[2], a[3])};
}

// byte offset of element (row, k) of a [128 x 64] K-major tile in core-matrix layout:
// core matrix (row/8, k/8) is 8 rows x 16 bytes; consecutive row groups 128 bytes apart (SBO),
// consecutive k groups 16 * 128 bytes apart (LBO)
__device__ __forceinline__ int tile_offset(int row, int k) {
    return ((k >> 3) * (kM / 8) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    // SM100 shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
    // version 1 [46,48), base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0) [61,64)
    const uint64_t lbo = (kM / 8) * 128;
    const uint64_t sbo = 128;
    return (static_cast<uint64_t>((saddr >> 4) & 0x3fff)) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: D F32, A/B BF16, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    const uint32_t no_mask = 0;  // no disabled output lanes
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(no_mask));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&out)[32]) {
    uint32_t v[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
          "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
          "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
          "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) out[j] = __uint_as_float(v[j]);
}

struct TcParams {
    int R, nb, nq, splits;
    const double* H;
    const double* axis[3];
    const RowDesc* rows;
    const int32_t* max_bin;
    const double* q;
    float* sinqd;
    float* bound;
    float* habs;
    int32_t* error_flag;
};

// grid: x = q tiles, y = row tiles, z = splits * 3 (K split, distance axis)
__global__ void __launch_bounds__(kThreadsTC, 1) debye_tc_kernel(TcParams P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* A_hi = smem;
    unsigned char* A_mid = smem + 1 * kTileBytes;
    unsigned char* A_lo = smem + 2 * kTileBytes;
    unsigned char* A_mag = smem + 3 * kTileBytes;
    unsigned char* B_hi = smem + 4 * kTileBytes;
    unsigned char* B_mid = smem + 5 * kTileBytes;
    unsigned char* B_lo = smem + 6 * kTileBytes;
    unsigned char* B_mag = smem + 7 * kTileBytes;
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail;
    __shared__ float s_ax[kKC];
    __shared__ float s_habs[kM];

    const int tid = threadIdx.x, warp = tid >> 5;
    const int m = tid & (kM - 1), half = tid >> 7;  // operand row / q column, half of the K chunk
    const int split = blockIdx.z / 3, g = blockIdx.z % 3;
    const int q0 = blockIdx.x * kN;
    const int r0 = blockIdx.y * kM;
    const int mb = *P.max_bin;
    const int per = debye_tc_split_bins(mb, P.splits);
    const int kb = split * per, ke = min(mb, kb + per);
    const double* axis = P.axis[g];

    // threads m and m + 128 stage row r0 + m of H and q value q0 + m of S (one half of a chunk each)
    const int r = r0 + m;
    const bool row_on = r < P.R && P.rows[r].group == g;
    if (!__syncthreads_or(row_on)) return;  // no row of this tile uses distance axis g
    float* out_v = P.sinqd + static_cast<size_t>(split) * P.R * P.nq;
    float* out_b = P.bound + static_cast<size_t>(split) * P.R * P.nq;
    if (kb >= ke) {
        // this split holds no bins: its partial sums are zero
        if (row_on && half == 0) {
            for (int j = 0; j < kN && q0 + j < P.nq; ++j) {
                out_v[static_cast<size_t>(r) * P.nq + q0 + j] = 0.f;
                out_b[static_cast<size_t>(r) * P.nq + q0 + j] = 0.f;
            }
            if (blockIdx.x == 0) P.habs[static_cast<size_t>(split) * P.R + r] = 0.f;
        }
        return;
    }
    const float qn = q0 + m < P.nq ? static_cast<float>(P.q[q0 + m]) : 0.f;
    const bool q_on = q0 + m < P.nq;
    const double* hrow = row_on ? P.H + static_cast<size_t>(r) * P.nb : nullptr;

    if (tid == 0) {
        s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    const uint32_t bar = smem_u32(&s_bar);

    float habs = 0.f;
    uint32_t parity = 0;
    bool first = true;
    for (int k0 = kb; k0 < ke; k0 += kKC) {
        if (tid < kKC) s_ax[tid] = k0 + tid < ke ? static_cast<float>(axis[k0 + tid]) : 0.f;
        __syncthreads();
        // ---- stage the operand tiles of this chunk: row m of A, column m of B, this thread's half ----
#pragma unroll 1
        for (int kg = half * (kKC / 16); kg < (half + 1) * (kKC / 16); ++kg) {
            float hv[8], sv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int b = k0 + kg * 8 + j;
                const float h = (row_on && b < ke) ? static_cast<float>(hrow[b]) : 0.f;
                habs += fabsf(h);
                hv[j] = h;
                float sc = 0.f;
                if (q_on && b < ke) {
                    const float x = qn * s_ax[kg * 8 + j];
                    sc = x < 1e-3f ? 1.f - x * x * (1.f / 6.f) : sinf(x) / x;
                }
                sv[j] = sc;
            }
            const int off = tile_offset(m, kg * 8);
            const Split8 a = split8(hv);
            *reinterpret_cast<uint4*>(A_hi + off) = a.hi;
            *reinterpret_cast<uint4*>(A_mid + off) = a.mid;
            *reinterpret_cast<uint4*>(A_lo + off) = a.lo;
            *reinterpret_cast<uint4*>(A_mag + off) = a.mag;
            const Split8 bs = split8(sv);
            *reinterpret_cast<uint4*>(B_hi + off) = bs.hi;
            *reinterpret_cast<uint4*>(B_mid + off) = bs.mid;
            *reinterpret_cast<uint4*>(B_lo + off) = bs.lo;
            *reinterpret_cast<uint4*>(B_mag + off) = bs.mag;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        // ---- issue the chunk's MMAs ----
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
            for (int ks = 0; ks < kKC / 16; ++ks) {
                const uint32_t koff = ks * 2 * (kM / 8) * 128;  // two k groups of 8 per K-step
                const uint64_t ah = smem_desc(smem_u32(A_hi) + koff), am = smem_desc(smem_u32(A_mid) + koff);
                const uint64_t al = smem_desc(smem_u32(A_lo) + koff), aa = smem_desc(smem_u32(A_mag) + koff);
                const uint64_t bh = smem_desc(smem_u32(B_hi) + koff), bm = smem_desc(smem_u32(B_mid) + koff);
                const uint64_t bl = smem_desc(smem_u32(B_lo) + koff), ba = smem_desc(smem_u32(B_mag) + koff);
                const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                mma_bf16(tmem, ah, bh, acc);
                mma_bf16(tmem + kColCorr, ah, bm, acc);
                mma_bf16(tmem + kColCorr, am, bh, 1u);
                mma_bf16(tmem + kColCorr, ah, bl, 1u);
                mma_bf16(tmem + kColCorr, al, bh, 1u);
                mma_bf16(tmem + kColCorr, am, bm, 1u);
                mma_bf16(tmem + kColBound, aa, ba, acc);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        first = false;
        // ---- wait until the MMAs have consumed the tiles ----
        if (!mbar_wait(bar, parity)) {
            if (tid == 0) s_fail = 1;
        }
        parity ^= 1u;
        __syncthreads();
        if (s_fail) break;
    }

    if (!s_fail) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // warp w reads TMEM lanes 32 (w % 4) .. +31 (its rows), the two halves split the q columns
        const uint32_t lane_base = static_cast<uint32_t>((warp & 3) * 32) << 16;
#pragma unroll 1
        for (int c0 = half * (kN / 2); c0 < (half + 1) * (kN / 2); c0 += 32) {
            float vm[32], vc[32], vb[32];
            tmem_ld32(tmem + lane_base + c0, vm);
            tmem_ld32(tmem + lane_base + kColCorr + c0, vc);
            tmem_ld32(tmem + lane_base + kColBound + c0, vb);
            if (row_on) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int qi = q0 + c0 + j;
                    if (qi < P.nq) {
                        out_v[static_cast<size_t>(r) * P.nq + qi] = vm[j] + vc[j];
                        out_b[static_cast<size_t>(r) * P.nq + qi] = vb[j];
                    }
                }
            }
        }
        if (half == 1) s_habs[m] = habs;
        __syncthreads();
        if (half == 0 && row_on && blockIdx.x == 0) P.habs[static_cast<size_t>(split) * P.R + r] = habs + s_habs[m];
    } else {
        // the MMAs of the timed-out chunk may still be running: wait for them (bounded) before
        // the tensor memory is released
        mbar_wait(bar, parity ^ 1u);
        if (tid == 0) atomicExch(P.error_flag, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

}  // namespace

size_t debye_tc_smem_bytes() { return 8 * static_cast<size_t>(kTileBytes) + 1024; }

int debye_tc_splits(int R, int bins, int nq, int sms, int groups) {
    const long long tiles = (long long)((nq + kN - 1) / kN) * ((R + kM - 1) / kM) * std::max(1, groups);
    const int chunks = std::max(1, (bins + kKC - 1) / kKC);
    long long s = (sms + tiles - 1) / std::max(1ll, tiles);
    s = std::max(1ll, std::min<long long>(s, std::min(64, chunks)));
    return (int)s;
}

bool debye_tc_launch(const TcArgs& A, cudaStream_t s) {
    static bool configured = false;
    const size_t smem = debye_tc_smem_bytes();
    if (!configured) {
        if (cudaFuncSetAttribute(debye_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return false;
        configured = true;
    }
    if (A.R <= 0 || A.nq <= 0 || A.splits <= 0) return false;
    TcParams P;
    P.R = A.R;
    P.nb = A.nb;
    P.nq = A.nq;
    P.splits = A.splits;
    P.H = A.H;
    P.axis[0] = A.axis0;
    P.axis[1] = A.axis1 ? A.axis1 : A.axis0;
    P.axis[2] = A.axis2 ? A.axis2 : A.axis0;
    P.rows = A.rows;
    P.max_bin = A.max_bin;
    P.q = A.q;
    P.sinqd = A.sinqd;
    P.bound = A.bound;
    P.habs = A.habs;
    P.error_flag = A.error_flag;
    dim3 grid((A.nq + kN - 1) / kN, (A.R + kM - 1) / kM, A.splits * 3);
    debye_tc_kernel<<<grid, kThreadsTC, smem, s>>>(P);
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace ausaxs_b200
