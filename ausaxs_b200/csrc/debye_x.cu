// Tensor-core Debye transform with exact integer accumulation over shared Taylor tables (sm_100a).
//
//   S_r(q) = sum_b H_r[b] sinc(q d_b)
//
// is the reference's sinc contraction (CompositeDistanceHistogramFFAvgBase.cpp:427-467).  A bin's
// distance lies in its bin: d_b = b w + (w / 2) u_b with |u_b| <= 1 (a weighted bin holds the mean of
// distances that round to b), so
//
//   sinc(q b w + q (w / 2) u) = sum_{k < K} C_k(b, q) u^k + R_K,   C_k(b, q) = c_k(q b w) (q w / 2)^k,
//   c_k(x) = sinc^(k)(x) / k!,   |R_K| <= (q w |u| / 2)^K / (K! (K + 1)),
//
// and S_r(q) = sum_{k, b} [H_r[b] u_b^k] C_k(b, q): a contraction over (k, b) whose right operand
// depends only on q, w and b -- one table serves every structure of a batch -- and whose left operand
// is the histogram row times powers of the in-bin offsets.
//
// Both operands are fixed-point numbers, one power-of-two scale per row (left) and a fixed scale 2 for
// the table, cut into six base-128 digits, the leading one signed (int8; Ozaki-style splitting).  tcgen05.mma
// kind::i8 adds the digit products of equal weight 2^-7(i+j+2) (i + j <= 5: 21 of the 36 pairs) into
// six s32 accumulators in tensor memory.  Integer accumulation is exact, so the value's error is the
// digit representation (2^-43 of a scale), the dropped pairs (2^-38.67 of the row scale per product)
// and the truncation R_K, each bounded per (row, q); the FP64 epilogue (debye.cu) adds the bounds up
// and recomputes a q value in FP64 only when they exceed the tolerance.
//
//   * tables (debye_x_table_kernel): for each q tile of 64 q values, chunk of 64 bins and order k, six
//     digit tiles [64 q x 64 bins] in the no-swizzle K-major core-matrix layout, contiguous (24 KiB),
//     so one bulk copy stages a (chunk, order) step; c_k from its power series below x = 2 and from
//     the product of the series of sin(x + t) and 1 / (x + t) above;
//   * contraction (debye_x_kernel): a CTA owns 128 rows x 64 q values of one split (a range of
//     chunks).  Per chunk the rows' H and u are staged in shared memory; per order k one thread
//     starts the table block's bulk copy, every thread digitises H u^k for half a chunk of one row
//     into six tiles [128 rows x 64 bins] and multiplies its staged values by u for the next order,
//     one thread issues the 42 MMAs (two K steps of 32) and commits them to an mbarrier.  Epilogue:
//     tcgen05.ld of the six accumulators, sum_s D_s 2^-7(s+2) times the scales in FP64.  Every wait is bounded; on timeout the kernel records an error flag,
//     waits (bounded) for its copies and MMAs, frees its tensor memory and returns, and the epilogue
//     takes FP64 for every q.
#include <algorithm>
#include <cmath>

#include "debye.cuh"

namespace ausaxs_b200 {
namespace {

constexpr int kXM = 128;                   // rows per CTA (UMMA M)
constexpr int kXN = kXQTile;               // q values per CTA (UMMA N)
constexpr int kXB = kXChunk;               // bins per chunk: two UMMA K steps of 32
constexpr int kXThreads = 256;
constexpr int kDigits = 6;
constexpr int kATile = kXM * kXB;          // one digit tile of the rows (8 KiB)
constexpr int kBTile = kXN * kXB;          // one digit tile of the table (4 KiB)
constexpr int kBBlock = kDigits * kBTile;  // one (q tile, chunk, order) block of the table (24 KiB)
constexpr int kXTmemCols = 512;            // six accumulators of 64 columns
constexpr unsigned kXSpin = 1u << 22;
constexpr int kMaxKSteps = 21000;          // |D_s| <= 6 * 128^2 per K element: s32-exact below 21,845

__constant__ double c_inv_fact[20] = {1.0,
                                      1.0,
                                      1.0 / 2,
                                      1.0 / 6,
                                      1.0 / 24,
                                      1.0 / 120,
                                      1.0 / 720,
                                      1.0 / 5040,
                                      1.0 / 40320,
                                      1.0 / 362880,
                                      1.0 / 3628800,
                                      1.0 / 39916800,
                                      1.0 / 479001600,
                                      1.0 / 6227020800.0,
                                      1.0 / 87178291200.0,
                                      1.0 / 1307674368000.0,
                                      1.0 / 20922789888000.0,
                                      1.0 / 355687428096000.0,
                                      1.0 / 6402373705728000.0,
                                      1.0 / 121645100408832000.0};

// byte offset of (row, k) in a K-major int8 tile of `rows` rows, no swizzle: core matrix (row / 8, k / 16)
// is 8 rows x 16 bytes; row groups 128 bytes apart (SBO), k groups rows * 16 bytes apart (LBO)
__host__ __device__ constexpr int xoff(int rows, int row, int k) {
    return ((k >> 4) * (rows / 8) + (row >> 3)) * 128 + (row & 7) * 16 + (k & 15);
}

__device__ __forceinline__ uint32_t xsmem(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t xdesc(uint32_t saddr, int rows) {
    // SM100 shared-memory matrix descriptor: start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46),
    // version 1 [46,48), base offset 0, layout SWIZZLE_NONE [61,64)
    const uint64_t lbo = static_cast<uint64_t>(rows / 8) * 128;
    const uint64_t sbo = 128;
    return (static_cast<uint64_t>((saddr >> 4) & 0x3fff)) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: D S32 [4,6) = 2, A S8 [7,10) = 1, B S8 [10,13) = 1, both K-major, N >> 3 at 17,
// M >> 4 at 24
constexpr uint32_t kXIdesc =
    (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kXN >> 3) << 17) | (static_cast<uint32_t>(kXM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    const uint32_t no_mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kXIdesc), "r"(accumulate), "r"(no_mask));
}

__device__ __forceinline__ void xbar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(xsmem(bar)) : "memory");
}

__device__ __forceinline__ void xbulk(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(xsmem(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     xsmem(dst)),
                 "l"(src), "r"(bytes), "r"(xsmem(bar))
                 : "memory");
}

__device__ __forceinline__ bool xwait(unsigned long long* bar, uint32_t parity) {
    const uint32_t a = xsmem(bar);
    for (unsigned it = 0; it < kXSpin; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld32i(uint32_t addr, int (&out)[32]) {
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
    for (int j = 0; j < 32; ++j) out[j] = static_cast<int>(v[j]);
}

// Six base-128 digits of X = rint(v), |v| < 127.5 * 2^35: X = sum_i d_i 2^(7 (5 - i)) with d_0 =
// floor(X / 2^35) in [-128, 127] and d_1..d_5 in [0, 127], each an int8.  rint through the FP64
// magic number 1.5 * 2^52, whose bit pattern then holds X in its low 52 bits.
__device__ __forceinline__ void digits6(double v, int (&d)[kDigits]) {
    const long long bits = __double_as_longlong(v + 6755399441055744.0);
    const unsigned lo = static_cast<unsigned>(bits);
    const int hi = static_cast<int>(bits >> 32) - 0x43380000;  // X >> 32
    d[5] = static_cast<int>(lo & 127u);
    d[4] = static_cast<int>((lo >> 7) & 127u);
    d[3] = static_cast<int>((lo >> 14) & 127u);
    d[2] = static_cast<int>((lo >> 21) & 127u);
    d[1] = static_cast<int>(__funnelshift_r(lo, static_cast<unsigned>(hi), 28) & 127u);
    d[0] = hi >> 3;
}

// c_k(x) = sinc^(k)(x) / k! for x >= 0; sx, cx = sin x, cos x
__device__ double sinc_coeff(double x, int k, double sx, double cx) {
    if (x < 2.0) {
        // sinc(x) = sum_n (-1)^n x^(2n) / (2n + 1)!, so c_k(x) = (1 / k!) sum_{2n >= k} (-1)^n x^(2n-k) /
        // ((2n - k)! (2n + 1)); the terms fall below 1e-28 of the first within 18 of them
        const int n0 = (k + 1) >> 1;
        int m = 2 * n0 - k;
        double t = m == 0 ? 1.0 : x;  // x^m / m!
        double s = 0;
        for (int n = n0; n < n0 + 18; ++n) {
            s += ((n & 1) ? -t : t) / (2 * n + 1);
            t *= x * x / ((m + 1) * (m + 2));
            m += 2;
        }
        return s * c_inv_fact[k];
    }
    // sin(x + t) = sum_m sin(x + m pi / 2) t^m / m!,  1 / (x + t) = sum_j (-1)^j t^j / x^(j+1)
    const double r = 1.0 / x;
    double s = 0, p = r;
    for (int j = 0; j <= k; ++j) {
        const int mm = k - j;
        const double sm = (mm & 1) ? ((mm & 2) ? -cx : cx) : ((mm & 2) ? -sx : sx);
        s += sm * c_inv_fact[mm] * p;
        p *= -r;
    }
    return s;
}

// grid (q tiles, chunks); thread item = (q in tile, 16-bin group, order)
__global__ void __launch_bounds__(256) debye_x_table_kernel(const double* q, int nq, double w, int nch, int K,
                                                            unsigned char* table, double* cpart) {
    __shared__ double s_cp[kXMaxOrder * 4][kXN];
    const int qt = blockIdx.x, c = blockIdx.y;
    const int nqp = gridDim.x * kXN;
    for (int item = threadIdx.x; item < kXN * 4 * K; item += blockDim.x) {
        const int qi = item % kXN, g = (item / kXN) % 4, k = item / (kXN * 4);
        const int qg = qt * kXN + qi;
        const double qv = qg < nq ? q[qg] : 0.0;
        const double hq = qv * w * 0.5;
        double hk = 1.0;
        for (int j = 0; j < k; ++j) hk *= hq;  // (q w / 2)^k
        uint32_t pack[kDigits][4];
#pragma unroll
        for (int j = 0; j < kDigits; ++j) pack[j][0] = pack[j][1] = pack[j][2] = pack[j][3] = 0;
        double asum = 0;
#pragma unroll 1
        for (int e = 0; e < 16; ++e) {
            const int b = c * kXB + g * 16 + e;
            double C = 0;
            if (qg < nq) {
                const double x = qv * (static_cast<double>(b) * w);
                double sx = 0, cx = 1;
                if (x >= 2.0) sincos(x, &sx, &cx);
                C = sinc_coeff(x, k, sx, cx) * hk;
            }
            asum += fabs(C);
            // C / 2 in fixed point with 42 fraction bits (|C| <= 1)
            int d[kDigits];
            digits6(C * 0x1p41, d);
#pragma unroll
            for (int j = 0; j < kDigits; ++j)
                pack[j][e >> 2] |= (static_cast<uint32_t>(d[j]) & 0xffu) << (8 * (e & 3));
        }
        unsigned char* blk = table + ((static_cast<size_t>(qt) * nch + c) * K + k) * kBBlock;
#pragma unroll
        for (int j = 0; j < kDigits; ++j)
            *reinterpret_cast<uint4*>(blk + j * kBTile + xoff(kXN, qi, g * 16)) =
                make_uint4(pack[j][0], pack[j][1], pack[j][2], pack[j][3]);
        s_cp[k * 4 + g][qi] = asum;
    }
    __syncthreads();
    for (int qi = threadIdx.x; qi < kXN; qi += blockDim.x) {
        double t = 0;
        for (int i = 0; i < 4 * K; ++i) t += s_cp[i][qi];
        cpart[static_cast<size_t>(c) * nqp + qt * kXN + qi] = t;
    }
}

struct XParams {
    const XRow* rows;
    int n_rows;
    const double* q;
    int nq;
    const unsigned char* table;
    int nch, K;
    double w;
    int cps;
    int32_t* error_flag;
};

// grid (q tiles, row tiles of 128, splits)
__global__ void __launch_bounds__(kXThreads, 1) debye_x_kernel(XParams P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* Abuf = smem;                     // kDigits tiles [128 rows x 64 bins]
    unsigned char* Bbuf = smem + kDigits * kATile;  // one table block: kDigits tiles [64 q x 64 bins]
    // the chunk's H u^k and u, [64 bins][128 rows] (consecutive rows in consecutive banks)
    double* s_hu = reinterpret_cast<double*>(smem + kDigits * kATile + kBBlock);
    double* s_u = s_hu + kXB * kXM;
    __shared__ __align__(8) unsigned long long bar_b, bar_m;
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail, s_nch;
    __shared__ double s_part[kXM];   // the second half's partial maximum, then the row's scale A
    __shared__ double s_hpart[kXM];  // the second half's partial sum |H|, then the row's sum
    __shared__ double s_mul[kXM];    // 2^42 / A: a value's fixed-point multiplier

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m = tid & (kXM - 1), half = tid >> 7;
    const int qt = blockIdx.x, z = blockIdx.z;
    const int row = blockIdx.y * kXM + m;
    XRow R{};
    if (row < P.n_rows) R = P.rows[row];
    const int mb = R.H ? *R.max_bin : 0;
    if (tid == 0) {
        s_nch = 0;
        s_fail = 0;
    }
    __syncthreads();
    if (half == 0 && mb > 0) atomicMax(&s_nch, (mb + kXB - 1) / kXB);
    __syncthreads();
    const int nch = min(s_nch, P.nch);
    const int c_lo = z * P.cps, c_hi = min(nch, c_lo + P.cps);
    const int q0 = qt * kXN;
    const int b_lo = c_lo * kXB, b_hi = min(c_hi * kXB, mb);  // this row's bins in the split
    if (c_lo >= c_hi) {
        // the split holds no bin of these rows: zero partial sums
        if (R.H && half == 0) {
            for (int j = 0; j < kXN && q0 + j < P.nq; ++j) R.out[z * R.out_z + q0 + j] = 0.0;
            if (qt == 0) R.e1[z * R.e_z] = R.e0[z * R.e_z] = R.habs[z * R.e_z] = 0.0;
        }
        return;
    }

    // ---- row scale: max over the split's bins of |H| max(1, |u|)^(K-1), and sum |H| ----
    const double two_w = 2.0 / P.w;
    double mx = 0, ha = 0;
    if (R.H && b_hi > b_lo) {
        const int mid = (b_lo + b_hi) >> 1;
        const int lo = half ? mid : b_lo, hi = half ? b_hi : mid;
        for (int b = lo; b < hi; ++b) {
            const double h = fabs(R.H[b]);
            const double u = fmax(1.0, fabs((R.axis[b] - b * P.w) * two_w));
            double f = h;
            for (int k = 1; k < P.K; ++k) f *= u;
            mx = fmax(mx, f);
            ha += h;
        }
    }
    if (half == 1) {
        s_part[m] = mx;
        s_hpart[m] = ha;
    }
    __syncthreads();
    if (half == 0) {
        mx = fmax(mx, s_part[m]);
        ha += s_hpart[m];
        double A = 0, mul = 0;
        if (mx > 0) {
            // A = 2^e > mx * 128 / 126: the leading digit stays within [-128, 127]
            const int e = ilogb(mx * (128.0 / 126.0) * (1.0 + 0x1p-30)) + 1;
            A = ldexp(1.0, e);
            mul = ldexp(1.0, 42 - e);
        }
        s_part[m] = A;
        s_hpart[m] = ha;
        s_mul[m] = mul;
    }
    if (tid == 0) {
        xbar_init(&bar_b);
        xbar_init(&bar_m);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(xsmem(&s_tmem)),
                     "r"(kXTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = s_tmem;
    const double mul = s_mul[m];
    const unsigned char* tq = P.table + static_cast<size_t>(qt) * P.nch * P.K * kBBlock;

    uint32_t pb = 0, pm = 0;
    bool first = true;
    int pending = 0;  // 1: a table copy may be in flight, 2: MMAs may be in flight
    for (int c = c_lo; c < c_hi; ++c) {
        // ---- the chunk's H (order 0) and u of row m, bins [32 half, 32 half + 32) ----
        // (the previous chunk's MMAs completed before the last barrier, so the buffers are free)
#pragma unroll 4
        for (int e = 0; e < 32; ++e) {
            const int bl = half * 32 + e, b = c * kXB + bl;
            double h = 0, u = 0;
            if (b < b_hi) {
                h = R.H[b];
                u = (R.axis[b] - b * P.w) * two_w;
            }
            s_hu[bl * kXM + m] = h * mul;  // H in units of 2^-42 A
            s_u[bl * kXM + m] = u;
        }
        for (int k = 0; k < P.K; ++k) {
            if (tid == 0) xbulk(Bbuf, tq + (static_cast<size_t>(c) * P.K + k) * kBBlock, kBBlock, &bar_b);
            // ---- digits of H u^k, then H u^(k+1) for the next order ----
#pragma unroll 1
            for (int g = 0; g < 2; ++g) {
                const int bl0 = half * 32 + g * 16;
                uint32_t pack[kDigits][4];
#pragma unroll
                for (int j = 0; j < kDigits; ++j) pack[j][0] = pack[j][1] = pack[j][2] = pack[j][3] = 0;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int i = (bl0 + e) * kXM + m;
                    const double v = s_hu[i];
                    s_hu[i] = v * s_u[i];
                    int d[kDigits];
                    digits6(v, d);
#pragma unroll
                    for (int j = 0; j < kDigits; ++j)
                        pack[j][e >> 2] |= (static_cast<uint32_t>(d[j]) & 0xffu) << (8 * (e & 3));
                }
#pragma unroll
                for (int j = 0; j < kDigits; ++j)
                    *reinterpret_cast<uint4*>(Abuf + j * kATile + xoff(kXM, m, bl0)) =
                        make_uint4(pack[j][0], pack[j][1], pack[j][2], pack[j][3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                if (!xwait(&bar_b, pb)) {
                    s_fail = 1;  // the copy may still be in flight
                } else {
                    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
                    for (int ks = 0; ks < kXB / 32; ++ks) {
                        const uint32_t ka = ks * 2 * (kXM / 8) * 128, kb = ks * 2 * (kXN / 8) * 128;
#pragma unroll
                        for (int s = 0; s < kDigits; ++s)
#pragma unroll
                            for (int i = 0; i <= s; ++i) {
                                const uint64_t da = xdesc(xsmem(Abuf + i * kATile) + ka, kXM);
                                const uint64_t db = xdesc(xsmem(Bbuf + (s - i) * kBTile) + kb, kXN);
                                mma_i8(tmem + s * kXN, da, db, (first && ks == 0 && i == 0) ? 0u : 1u);
                            }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     xsmem(&bar_m))
                                 : "memory");
                }
            }
            __syncthreads();
            if (s_fail) {
                pending = 1;
                break;
            }
            pb ^= 1u;
            first = false;
            if (!xwait(&bar_m, pm)) {
                if (tid == 0) s_fail = 2;
            }
            pm ^= 1u;
            __syncthreads();
            if (s_fail) {
                pending = 2;
                break;
            }
        }
        if (s_fail) break;
    }

    if (!s_fail) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows), columns 32 (w / 4) .. + 31 (q values)
        const int rm = (warp & 3) * 32 + lane;
        const uint32_t lane_base = static_cast<uint32_t>((warp & 3) * 32) << 16;
        const int cb = (warp >> 2) * 32;
        double acc[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] = 0;
#pragma unroll 1
        for (int s = 0; s < kDigits; ++s) {
            int v[32];
            tmem_ld32i(tmem + lane_base + s * kXN + cb, v);
            const double wgt = ldexp(1.0, -7 * (s + 2));
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[j] += static_cast<double>(v[j]) * wgt;
        }
        const int rrow = blockIdx.y * kXM + rm;
        if (rrow < P.n_rows) {
            const XRow Rr = P.rows[rrow];
            if (Rr.H) {
                const double A2 = s_part[rm] * 2.0;  // row scale times the table's scale
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int qi = q0 + cb + j;
                    if (qi < P.nq) Rr.out[z * Rr.out_z + qi] = acc[j] * A2;
                }
                if (qt == 0 && cb == 0) {
                    // per element: digits of H u^k within 2^-43 A (one rounding of the fixed-point
                    // value; the staged H u^k carry 2^-52 relative more), of C_k within 2^-42; dropped
                    // digit pairs (i + j >= 6) below 2^-38.67 A; sum_k |H u^k| <= K 1.01^(K-1) sum |H|
                    const double nK = static_cast<double>(c_hi - c_lo) * kXB * P.K;
                    const double hs = s_hpart[rm];
                    Rr.e1[z * Rr.e_z] = s_part[rm] * 0x1p-42;
                    Rr.e0[z * Rr.e_z] = s_part[rm] * nK * 0x1p-38 + 0x1p-41 * 1.1 * P.K * hs;
                    Rr.habs[z * Rr.e_z] = hs;
                }
            }
        }
    } else {
        // bounded waits for the copies and MMAs this CTA may still have in flight
        if (pending == 1) xwait(&bar_b, pb);
        if (pending == 2) xwait(&bar_m, pm ^ 1u);
        if (tid == 0) atomicExch(P.error_flag, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kXTmemCols));
}

}  // namespace

int debye_x_order(double qmax, double w) {
    const double x = std::max(0.0, qmax) * w * 0.5;
    double f = 1;  // K!
    for (int K = 1; K <= kXMaxOrder; ++K) {
        f *= K;
        if (K >= 2 && std::pow(x, K) / (f * (K + 1)) <= 0x1p-32) return K;
    }
    return kXMaxOrder;
}

double debye_x_trunc(int K, double w) {
    double f = 1;
    for (int k = 2; k <= K; ++k) f *= k;
    return std::pow(w * 0.5 * 1.01, K) / (f * (K + 1));
}

int debye_x_max_chunks(int K) { return std::max(1, kMaxKSteps / (kXB * std::max(1, K))); }

size_t debye_x_table_bytes(int nq, int nch, int K) {
    return static_cast<size_t>((nq + kXN - 1) / kXN) * nch * K * kBBlock;
}

size_t debye_x_cpart_doubles(int nq, int nch) { return static_cast<size_t>((nq + kXN - 1) / kXN) * kXN * nch; }

size_t debye_x_smem_bytes() {
    return static_cast<size_t>(kDigits) * kATile + kBBlock + 2 * sizeof(double) * kXB * kXM + 1024;
}

void debye_x_table_launch(const double* q, int nq, double w, int nch, int K, unsigned char* table, double* cpart,
                          cudaStream_t s) {
    if (nq <= 0 || nch <= 0) return;
    debye_x_table_kernel<<<dim3((nq + kXN - 1) / kXN, nch), 256, 0, s>>>(q, nq, w, nch, K, table, cpart);
}

bool debye_x_launch(const XRow* rows, int n_rows, const double* q, int nq, const unsigned char* table, int nch, int K,
                    double w, int cps, int splits, int32_t* error_flag, cudaStream_t s) {
    static bool configured = false;
    const size_t smem = debye_x_smem_bytes();
    if (!configured) {
        if (cudaFuncSetAttribute(debye_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return false;
        configured = true;
    }
    if (n_rows <= 0 || nq <= 0 || splits <= 0 || cps <= 0 || K < 1 || K > kXMaxOrder) return false;
    if (static_cast<long long>(cps) * kXB * K > kMaxKSteps) return false;
    XParams P;
    P.rows = rows;
    P.n_rows = n_rows;
    P.q = q;
    P.nq = nq;
    P.table = table;
    P.nch = nch;
    P.K = K;
    P.w = w;
    P.cps = cps;
    P.error_flag = error_flag;
    const dim3 grid((nq + kXN - 1) / kXN, (n_rows + kXM - 1) / kXM, splits);
    debye_x_kernel<<<grid, kXThreads, smem, s>>>(P);
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace ausaxs_b200
