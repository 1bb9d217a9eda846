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
//     digit tiles [64 q x 64 bins] in the no-swizzle K-major core-matrix layout, contiguous (24 KiB);
//     c_k from its power series below x = 2 and from the product of the series of sin(x + t) and
//     1 / (x + t) above.  Rebuilt only when the q values change (debye_x_qcheck_kernel);
//   * rows (debye_x_rowstat_kernel, debye_x_digits_kernel): each row's power-of-two scale and bound
//     terms, then for every (M tile of 128 rows, chunk, order) six digit tiles [128 rows x 64 bins]
//     of H u^k (48 KiB, contiguous), made once and read by every q tile;
//   * contraction (debye_x_kernel): a CTA owns 128 rows x 64 q values of one split (a range of
//     chunks).  One thread streams the split's (chunk, order) steps through two stages of shared
//     memory by bulk copies of both digit blocks and issues each step's 42 MMAs (two K steps of 32)
//     when its copies land, so the copy of the next step overlaps them.  Epilogue: tcgen05.ld of the
//     six accumulators, sum_s D_s 2^-7(s+2) times the scales in FP64.  Every wait is bounded; on
//     timeout the kernel waits (bounded) for what it has in flight, frees its tensor memory and
//     records an error flag, and the epilogue then takes FP64 for every q.
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

// 1 / (2n + 1) and 1 / ((m + 1)(m + 2)) for the power series of c_k
__constant__ double c_inv_odd[32] = {
    1.0,        1.0 / 3,  1.0 / 5,  1.0 / 7,  1.0 / 9,  1.0 / 11, 1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19, 1.0 / 21,
    1.0 / 23,   1.0 / 25, 1.0 / 27, 1.0 / 29, 1.0 / 31, 1.0 / 33, 1.0 / 35, 1.0 / 37, 1.0 / 39, 1.0 / 41, 1.0 / 43,
    1.0 / 45,   1.0 / 47, 1.0 / 49, 1.0 / 51, 1.0 / 53, 1.0 / 55, 1.0 / 57, 1.0 / 59, 1.0 / 61, 1.0 / 63};
__constant__ double c_inv_pair[48] = {
    1.0 / 2,    1.0 / 6,    1.0 / 12,   1.0 / 20,   1.0 / 30,   1.0 / 42,   1.0 / 56,   1.0 / 72,
    1.0 / 90,   1.0 / 110,  1.0 / 132,  1.0 / 156,  1.0 / 182,  1.0 / 210,  1.0 / 240,  1.0 / 272,
    1.0 / 306,  1.0 / 342,  1.0 / 380,  1.0 / 420,  1.0 / 462,  1.0 / 506,  1.0 / 552,  1.0 / 600,
    1.0 / 650,  1.0 / 702,  1.0 / 756,  1.0 / 812,  1.0 / 870,  1.0 / 930,  1.0 / 992,  1.0 / 1056,
    1.0 / 1122, 1.0 / 1190, 1.0 / 1260, 1.0 / 1332, 1.0 / 1406, 1.0 / 1482, 1.0 / 1560, 1.0 / 1640,
    1.0 / 1722, 1.0 / 1806, 1.0 / 1892, 1.0 / 1980, 1.0 / 2070, 1.0 / 2162, 1.0 / 2256, 1.0 / 2352};

// c_k(x) = sinc^(k)(x) / k! for x >= 0; sx, cx = sin x, cos x
__device__ double sinc_coeff(double x, int k, double sx, double cx) {
    if (x < 2.0) {
        // sinc(x) = sum_n (-1)^n x^(2n) / (2n + 1)!, so c_k(x) = (1 / k!) sum_{2n >= k} (-1)^n x^(2n-k) /
        // ((2n - k)! (2n + 1)); with x < 2 the terms fall below 1e-20 of the first within 16 of them
        const int n0 = (k + 1) >> 1;
        int m = 2 * n0 - k;
        double t = m == 0 ? 1.0 : x;  // x^m / m!
        const double x2 = x * x;
        double s = 0;
#pragma unroll 4
        for (int n = n0; n < n0 + 16; ++n) {
            s += ((n & 1) ? -t : t) * c_inv_odd[n];
            t *= x2 * c_inv_pair[m];
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

// flags[0] = 1 when q differs bit for bit from the q the tables were made for (then copied there)
__global__ void debye_x_qcheck_kernel(const double* q, int nq, double* q_cached, int32_t* flags) {
    int diff = 0;
    for (int i = threadIdx.x; i < nq; i += blockDim.x)
        diff |= __double_as_longlong(q[i]) != __double_as_longlong(q_cached[i]);
    diff = __syncthreads_or(diff);
    if (diff)
        for (int i = threadIdx.x; i < nq; i += blockDim.x) q_cached[i] = q[i];
    if (threadIdx.x == 0) flags[0] = diff;
}

// grid (q tiles, chunks); thread = (q in tile, 16-bin group): sin and cos of its 16 arguments once,
// then every order's digits
__global__ void __launch_bounds__(256) debye_x_table_kernel(const double* q, int nq, double w, int nch, int K,
                                                            unsigned char* table, double* cpart,
                                                            const int32_t* flags) {
    if (!flags[0]) return;  // the tables hold this q grid already
    __shared__ double s_cp[4][kXN];
    const int qt = blockIdx.x, c = blockIdx.y;
    const int nqp = gridDim.x * kXN;
    const int qi = threadIdx.x % kXN, g = threadIdx.x / kXN;  // 256 threads: 64 q x 4 groups
    const int qg = qt * kXN + qi;
    const double qv = qg < nq ? q[qg] : 0.0;
    const double hq = qv * w * 0.5;
    double xs[16], sn[16], cs[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        xs[e] = qv * (static_cast<double>(c * kXB + g * 16 + e) * w);
        sn[e] = 0;
        cs[e] = 1;
        if (xs[e] >= 2.0) sincos(xs[e], &sn[e], &cs[e]);
    }
    double asum = 0, hk = 1.0;  // hk = (q w / 2)^k
    for (int k = 0; k < K; ++k) {
        uint32_t pack[kDigits][4];
#pragma unroll
        for (int j = 0; j < kDigits; ++j) pack[j][0] = pack[j][1] = pack[j][2] = pack[j][3] = 0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const double C = qg < nq ? sinc_coeff(xs[e], k, sn[e], cs[e]) * hk : 0.0;
            asum += fabs(C);
            int d[kDigits];
            digits6(C * 0x1p41, d);  // C / 2 in fixed point with 42 fraction bits (|C| <= 1)
#pragma unroll
            for (int j = 0; j < kDigits; ++j)
                pack[j][e >> 2] |= (static_cast<uint32_t>(d[j]) & 0xffu) << (8 * (e & 3));
        }
        unsigned char* blk = table + ((static_cast<size_t>(qt) * nch + c) * K + k) * kBBlock;
#pragma unroll
        for (int j = 0; j < kDigits; ++j)
            *reinterpret_cast<uint4*>(blk + j * kBTile + xoff(kXN, qi, g * 16)) =
                make_uint4(pack[j][0], pack[j][1], pack[j][2], pack[j][3]);
        hk *= hq;
    }
    s_cp[g][qi] = asum;
    __syncthreads();
    if (threadIdx.x < kXN)
        cpart[static_cast<size_t>(c) * nqp + qt * kXN + threadIdx.x] =
            s_cp[0][threadIdx.x] + s_cp[1][threadIdx.x] + s_cp[2][threadIdx.x] + s_cp[3][threadIdx.x];
}

// One warp per row: its scale A = 2^e > max_b |H| max(1, |u|)^(K-1) * 128 / 126 (row_scale[r]) and, per
// split, sum |H| and the bound terms of its digit arithmetic (debye_x_kernel's epilogue):
//   digits of H u^k within 2^-42 A (one rounding of the fixed-point value; the FP64 products H u^k
//   add 2^-52 relative), of C_k within 2^-42 -- e1 = 2^-42 A multiplies sum |C_k(b, q)|;
//   dropped digit pairs (i + j >= 6) below 2^-38.67 A per product and sum_k |H u^k| <= K 1.01^(K-1)
//   sum |H| -- e0 = 2^-38 A n_K + 2^-41 1.1 K sum |H|, n_K the split's products of the row.
__global__ void debye_x_rowstat_kernel(const XRow* rows, int n_rows, double w, int K, int cps, int splits,
                                       double* row_scale) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= n_rows) return;
    const XRow R = rows[r];
    if (!R.H) {
        if (lane == 0) row_scale[r] = 0;
        return;
    }
    const int mb = *R.max_bin;
    const double two_w = 2.0 / w;
    double mx = 0;
    for (int b = lane; b < mb; b += 32) {
        const double u = fmax(1.0, fabs((R.axis[b] - b * w) * two_w));
        double f = fabs(R.H[b]);
        for (int k = 1; k < K; ++k) f *= u;
        mx = fmax(mx, f);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    double A = 0;
    if (mx > 0) A = ldexp(1.0, ilogb(mx * (128.0 / 126.0) * (1.0 + 0x1p-30)) + 1);
    if (lane == 0) row_scale[r] = A;
    const int span = cps * kXB;
    for (int z = 0; z < splits; ++z) {
        const int b0 = z * span, b1 = min(mb, b0 + span);
        double hs = 0;
        for (int b = b0 + lane; b < b1; b += 32) hs += fabs(R.H[b]);
        for (int o = 16; o > 0; o >>= 1) hs += __shfl_xor_sync(0xffffffffu, hs, o);
        if (lane == 0) {
            const double nK = b1 > b0 ? static_cast<double>((b1 - b0 + kXB - 1) / kXB) * kXB * K : 0.0;
            R.e1[z * R.e_z] = b1 > b0 ? A * 0x1p-42 : 0.0;
            R.e0[z * R.e_z] = A * nK * 0x1p-38 + 0x1p-41 * 1.1 * K * hs;
            R.habs[z * R.e_z] = hs;
        }
    }
}

// chunks of bins an M tile needs: the largest of its rows' ceil(max_bin / 64) (CTA-wide, via shared memory)
__device__ int tile_chunks(const XRow* rows, int n_rows, int tile, int* s_n) {
    if (threadIdx.x == 0) *s_n = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < kXM; i += blockDim.x) {
        const int r = tile * kXM + i;
        if (r < n_rows && rows[r].H) atomicMax(s_n, (*rows[r].max_bin + kXB - 1) / kXB);
    }
    __syncthreads();
    return *s_n;
}

// grid (M tiles, chunks): the digit tiles of H u^k for every order k of one (M tile, chunk), written in
// the UMMA layout to adig + tile_off[tile] + (chunk K + k) 48 KiB
__global__ void __launch_bounds__(kXThreads) debye_x_digits_kernel(const XRow* rows, int n_rows, double w, int K,
                                                                   const double* row_scale,
                                                                   const long long* tile_off, unsigned char* adig) {
    constexpr int kPitch = kXM + 1;  // [bin][row], consecutive rows in consecutive banks
    extern __shared__ __align__(16) unsigned char dsm[];
    double* s_p = reinterpret_cast<double*>(dsm);  // H u^k in units of 2^-42 A
    double* s_u = s_p + kXB * kPitch;
    __shared__ const double* s_h[kXM];
    __shared__ const double* s_ax[kXM];
    __shared__ double s_mul[kXM];
    __shared__ int s_mb[kXM];
    __shared__ int s_n;
    const int tile = blockIdx.x, c = blockIdx.y;
    if (c >= tile_chunks(rows, n_rows, tile, &s_n)) return;
    for (int i = threadIdx.x; i < kXM; i += blockDim.x) {
        const int r = tile * kXM + i;
        const bool on = r < n_rows && rows[r].H && row_scale[r] > 0;
        s_h[i] = on ? rows[r].H : nullptr;
        s_ax[i] = on ? rows[r].axis : nullptr;
        s_mb[i] = on ? *rows[r].max_bin : 0;
        s_mul[i] = on ? 0x1p42 / row_scale[r] : 0.0;
    }
    __syncthreads();
    const double two_w = 2.0 / w;
    for (int i = threadIdx.x; i < kXM * kXB; i += blockDim.x) {
        const int rr = i / kXB, bl = i - rr * kXB, b = c * kXB + bl;
        double h = 0, u = 0;
        if (b < s_mb[rr]) {
            h = s_h[rr][b] * s_mul[rr];
            u = (s_ax[rr][b] - b * w) * two_w;
        }
        s_p[bl * kPitch + rr] = h;
        s_u[bl * kPitch + rr] = u;
    }
    __syncthreads();
    const int m = threadIdx.x & (kXM - 1), half = threadIdx.x >> 7;
    unsigned char* base = adig + tile_off[tile] + static_cast<size_t>(c) * K * (kDigits * kATile);
    for (int k = 0; k < K; ++k) {
        unsigned char* blk = base + static_cast<size_t>(k) * (kDigits * kATile);
#pragma unroll 1
        for (int g = 0; g < 2; ++g) {
            const int bl0 = half * 32 + g * 16;
            uint32_t pack[kDigits][4];
#pragma unroll
            for (int j = 0; j < kDigits; ++j) pack[j][0] = pack[j][1] = pack[j][2] = pack[j][3] = 0;
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                const int i = (bl0 + e) * kPitch + m;
                const double v = s_p[i];
                s_p[i] = v * s_u[i];
                int d[kDigits];
                digits6(v, d);
#pragma unroll
                for (int j = 0; j < kDigits; ++j)
                    pack[j][e >> 2] |= (static_cast<uint32_t>(d[j]) & 0xffu) << (8 * (e & 3));
            }
#pragma unroll
            for (int j = 0; j < kDigits; ++j)
                *reinterpret_cast<uint4*>(blk + j * kATile + xoff(kXM, m, bl0)) =
                    make_uint4(pack[j][0], pack[j][1], pack[j][2], pack[j][3]);
        }
    }
}

struct XParams {
    const XRow* rows;
    int n_rows;
    int nq;
    const unsigned char* table;
    const unsigned char* adig;
    const long long* tile_off;
    const double* row_scale;
    int nch, K, cps;
    int32_t* error_flag;
};

// grid (q tiles, M tiles, splits).  One thread streams the (chunk, order) steps of the split through
// two stages of shared memory (bulk copies of the rows' and the table's digit blocks, 72 KiB a stage)
// and issues each step's 42 MMAs as soon as its copies land; the copy of step t + 1 overlaps the MMAs of
// step t.  Then every warp reads its TMEM lanes and writes the FP64 values.
__global__ void __launch_bounds__(kXThreads, 1) debye_x_kernel(XParams P) {
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int kABlock = kDigits * kATile;  // 48 KiB
    constexpr int kStage = kABlock + kBBlock;  // 72 KiB
    __shared__ __align__(8) unsigned long long bar_full[2], bar_mma[2];
    __shared__ uint32_t s_tmem;
    __shared__ int s_fail, s_n;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int qt = blockIdx.x, tile = blockIdx.y, z = blockIdx.z;
    const int q0 = qt * kXN;
    const int nch = min(tile_chunks(P.rows, P.n_rows, tile, &s_n), P.nch);
    const int c_lo = z * P.cps, c_hi = min(nch, c_lo + P.cps);
    const int n_it = c_hi > c_lo ? (c_hi - c_lo) * P.K : 0;
    if (n_it == 0) {
        // the split holds no bin of these rows: zero partial sums
        for (int i = tid; i < kXM; i += blockDim.x) {
            const int r = tile * kXM + i;
            if (r < P.n_rows && P.rows[r].H) {
                const XRow R = P.rows[r];
                for (int j = 0; j < kXN && q0 + j < P.nq; ++j) R.out[z * R.out_z + q0 + j] = 0.0;
            }
        }
        return;
    }
    if (tid == 0) {
        s_fail = 0;
        for (int st = 0; st < 2; ++st) {
            xbar_init(&bar_full[st]);
            xbar_init(&bar_mma[st]);
        }
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

    if (tid == 0) {
        const unsigned char* abase = P.adig + P.tile_off[tile];
        const unsigned char* bbase = P.table + static_cast<size_t>(qt) * P.nch * P.K * kBBlock;
        auto issue = [&](int it) {
            const int st = it & 1;
            const size_t step = static_cast<size_t>(c_lo) * P.K + it;  // chunk * K + order
            unsigned char* dst = smem + st * kStage;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(xsmem(&bar_full[st])),
                         "r"(kStage)
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             xsmem(dst)),
                         "l"(abase + step * kABlock), "r"(kABlock), "r"(xsmem(&bar_full[st]))
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             xsmem(dst + kABlock)),
                         "l"(bbase + step * kBBlock), "r"(kBBlock), "r"(xsmem(&bar_full[st]))
                         : "memory");
        };
        int issued = 0, landed = 0, committed = 0, retired = 0;
        bool ok = true;
        issue(0);
        issued = 1;
        for (int it = 0; it < n_it && ok; ++it) {
            const int st = it & 1;
            if (it + 1 < n_it) {
                // stage (it + 1) & 1 was read by the MMAs of step it - 1
                if (it >= 1) {
                    ok = xwait(&bar_mma[(it - 1) & 1], ((it - 1) >> 1) & 1);
                    if (!ok) break;
                    retired = it;
                }
                issue(it + 1);
                issued = it + 2;
            }
            ok = xwait(&bar_full[st], (it >> 1) & 1);
            if (!ok) break;
            landed = it + 1;
            asm volatile("tcgen05.fence::after_thread_sync;");
            unsigned char* A = smem + st * kStage;
            unsigned char* B = A + kABlock;
#pragma unroll 1
            for (int ks = 0; ks < kXB / 32; ++ks) {
                const uint32_t ka = ks * 2 * (kXM / 8) * 128, kb = ks * 2 * (kXN / 8) * 128;
#pragma unroll
                for (int s = 0; s < kDigits; ++s)
#pragma unroll
                    for (int i = 0; i <= s; ++i) {
                        const uint64_t da = xdesc(xsmem(A + i * kATile) + ka, kXM);
                        const uint64_t db = xdesc(xsmem(B + (s - i) * kBTile) + kb, kXN);
                        mma_i8(tmem + s * kXN, da, db, (it == 0 && ks == 0 && i == 0) ? 0u : 1u);
                    }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             xsmem(&bar_mma[st]))
                         : "memory");
            committed = it + 1;
        }
        if (ok) {
            // the last commit completes after every earlier MMA
            ok = xwait(&bar_mma[(n_it - 1) & 1], ((n_it - 1) >> 1) & 1);
            if (ok) retired = n_it;
        }
        if (!ok) {
            // bounded waits for what may still be in flight, then report
            for (int it = landed; it < issued; ++it) xwait(&bar_full[it & 1], (it >> 1) & 1);
            if (committed > retired) xwait(&bar_mma[(committed - 1) & 1], ((committed - 1) >> 1) & 1);
            s_fail = 1;
        }
    }
    __syncthreads();

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
        const int r = tile * kXM + rm;
        if (r < P.n_rows) {
            const XRow R = P.rows[r];
            if (R.H) {
                const double A2 = P.row_scale[r] * 2.0;  // row scale times the table's scale
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int qi = q0 + cb + j;
                    if (qi < P.nq) R.out[z * R.out_z + qi] = acc[j] * A2;
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(P.error_flag, 1);
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

size_t debye_x_block_bytes() { return static_cast<size_t>(kDigits) * kATile; }

bool debye_x_enqueue(const XPlan& X, const double* q, cudaStream_t s) {
    static bool configured = false;
    const size_t smem_mma = 2 * (static_cast<size_t>(kDigits) * kATile + kBBlock);
    const size_t smem_dig = 2 * sizeof(double) * kXB * (kXM + 1);
    if (!configured) {
        if (cudaFuncSetAttribute(debye_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_mma) !=
                cudaSuccess ||
            cudaFuncSetAttribute(debye_x_digits_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_dig) !=
                cudaSuccess)
            return false;
        configured = true;
    }
    if (X.n_rows <= 0 || X.nq <= 0 || X.splits <= 0 || X.cps <= 0 || X.K < 1 || X.K > kXMaxOrder) return false;
    if (static_cast<long long>(X.cps) * kXB * X.K > kMaxKSteps) return false;
    const int nqt = (X.nq + kXN - 1) / kXN, tiles = (X.n_rows + kXM - 1) / kXM;
    debye_x_qcheck_kernel<<<1, 256, 0, s>>>(q, X.nq, X.q_cached, X.flags);
    debye_x_table_kernel<<<dim3(nqt, X.nch), 256, 0, s>>>(q, X.nq, X.w, X.nch, X.K, X.table, X.cpart, X.flags);
    debye_x_rowstat_kernel<<<(X.n_rows + 7) / 8, 256, 0, s>>>(X.rows, X.n_rows, X.w, X.K, X.cps, X.splits,
                                                               X.row_scale);
    debye_x_digits_kernel<<<dim3(tiles, X.nch), kXThreads, smem_dig, s>>>(X.rows, X.n_rows, X.w, X.K, X.row_scale,
                                                                          X.tile_off, X.adig);
    XParams P;
    P.rows = X.rows;
    P.n_rows = X.n_rows;
    P.nq = X.nq;
    P.table = X.table;
    P.adig = X.adig;
    P.tile_off = X.tile_off;
    P.row_scale = X.row_scale;
    P.nch = X.nch;
    P.K = X.K;
    P.cps = X.cps;
    P.error_flag = X.flags + 1;
    debye_x_kernel<<<dim3(nqt, tiles, X.splits), kXThreads, smem_mma, s>>>(P);
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace ausaxs_b200
