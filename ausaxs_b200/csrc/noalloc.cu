// Allocation-free Simple (weighted) histogram: the HistogramManagerMT path of ausaxs_gpu_histogram
// with every temporary in one file-scope device array instead of memory obtained at run time.
//
// Who needs this: callers that must not allocate device memory while they run -- for example code
// inside a memory-pool-managed or real-time section, an embedding application that forbids
// cudaMalloc after start-up (allocation can synchronise the device and stall other streams), or a
// framework that accounts for every device byte itself.  They pass device inputs and device outputs
// and get the histogram with no cudaMalloc, cudaFree or allocating library call.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxBins bins (the scratch array is sized for it: 591,104 bytes, about 577 KiB,
//     held on every device that loads this library until the process exits);
//   * all calls share the one array and it keeps the last call's contents (everything that must
//     start at zero is cleared by the call itself); calls that overlap on the GPU -- on different
//     streams, or from different host threads -- race on it and give wrong results, so serialise
//     the calls on one stream or order them with events;
//   * the array's device address belongs to the CUDA context that loaded this module.  The first
//     call in a context (per device, per context: a context created again after cudaDeviceReset
//     counts as new) looks the address up with cudaGetSymbolAddress and caches it under the
//     context's unique id; make that first call before any stream capture.
#include <cuda.h>  // CUcontext and the driver entry point types only; libcuda is not linked

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ausaxs_b200.h"
#include "finalize.cuh"
#include "pairhist.cuh"

namespace ausaxs_b200 {
void set_last_error(const char* msg);  // capi.cu

namespace {

constexpr int kNoAllocMaxBins = 8192;
constexpr int kNoAllocTile = 256;
constexpr size_t kJobBytes = 1024;  // three PairJob records
constexpr size_t kMiscBytes = 256;  // tile counters, overflow, weight scale, self sums
constexpr size_t kSlotBytes = 3ull * kNoAllocMaxBins * 8;  // counts, offset sums, weight sums of one job
constexpr size_t kScratchBytes = kJobBytes + kMiscBytes + 3 * kSlotBytes;

static_assert(kScratchBytes == 591104, "the documented scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device addresses of the scratch array, one per (device, context).  The context is identified by
// cuCtxGetId, which is unique for the life of the process (a context created again at the same
// handle gets a new id), reached through cudaGetDriverEntryPoint so that the library needs no link
// against the driver library.  Where the driver does not provide it, the device alone is the key.
struct ScratchAddr {
    struct Entry {
        int dev;
        unsigned long long ctx_id;
        void* ptr;
    };
    std::mutex m;
    std::vector<Entry> entries;
    bool resolved = false;
    CUresult (*ctx_get_current)(CUcontext*) = nullptr;
    CUresult (*ctx_get_id)(CUcontext, unsigned long long*) = nullptr;
};
ScratchAddr g_addr;

// The current context's id (0 when it cannot be determined).  Called with g_addr.m held.
unsigned long long current_context_id() {
    if (!g_addr.resolved) {
        g_addr.resolved = true;
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            g_addr.ctx_get_current = reinterpret_cast<CUresult (*)(CUcontext*)>(f1);
            g_addr.ctx_get_id = reinterpret_cast<CUresult (*)(CUcontext, unsigned long long*)>(f2);
        }
        cudaGetLastError();  // a failed lookup leaves nothing behind for the caller
    }
    if (!g_addr.ctx_get_current || !g_addr.ctx_get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (g_addr.ctx_get_current(&c) != CUDA_SUCCESS || !c) return 0;
    if (g_addr.ctx_get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Clears the scratch accumulators and writes the job table (passed by value, so no host copy).
struct NoAllocInit {
    PairJob jobs[3];
    int n_jobs;
    size_t clear_words;  // u64 words from the start of the misc block
};

__global__ void noalloc_init_kernel(NoAllocInit init) {
    unsigned char* base = g_noalloc_scratch;
    if (blockIdx.x == 0 && threadIdx.x < init.n_jobs) reinterpret_cast<PairJob*>(base)[threadIdx.x] = init.jobs[threadIdx.x];
    unsigned long long* z = reinterpret_cast<unsigned long long*>(base + kJobBytes);
    for (size_t k = blockIdx.x * blockDim.x + threadIdx.x; k < init.clear_words; k += gridDim.x * blockDim.x) z[k] = 0;
}

__global__ void noalloc_copy_u64(const unsigned long long* src, unsigned long long* dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = *src;
}

int fail(int code, const char* msg) {
    set_last_error(msg);  // read back with ausaxs_gpu_last_error()
    return code;
}

}  // namespace
}  // namespace ausaxs_b200

using namespace ausaxs_b200;

extern "C" int ausaxs_gpu_histogram_mt_noalloc(const float* atoms, int32_t n_atoms, const float* waters, int32_t n_waters,
                                               double bin_width, int32_t bin_count, int32_t weighted_bins,
                                               double* hist_out, int32_t* max_bin_out,
                                               unsigned long long* overflow_out, void* stream) {
    if (n_atoms < 0 || n_waters < 0 || (n_atoms && !atoms) || (n_waters && !waters) || !hist_out || !max_bin_out)
        return fail(AUSAXS_ERR_ARGUMENT, "invalid argument");
    if (!(bin_width > 0) || bin_count < 11)
        return fail(AUSAXS_ERR_ARGUMENT, "bin_width must be positive and bin_count at least 11");
    if (bin_count > kNoAllocMaxBins)
        return fail(AUSAXS_ERR_CAPACITY, "bin_count exceeds the allocation-free limit of 8192 bins");
    // an error left behind by an earlier, unrelated call must not be reported as this call's
    cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return fail(AUSAXS_ERR_CUDA, "no current CUDA device");
    // make the device's primary context current (initialised if it was not; a no-op when it already
    // is) so that the context id below is the one the launches use
    if (cudaSetDevice(dev) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, "cannot initialise the CUDA context");
    void* base_ptr = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_addr.m);
        const unsigned long long ctx_id = current_context_id();
        for (const auto& e : g_addr.entries)
            if (e.dev == dev && e.ctx_id == ctx_id) base_ptr = e.ptr;
        if (!base_ptr) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
            g_addr.entries.push_back({dev, ctx_id, p});
            base_ptr = p;
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(base_ptr);
    const int nb = bin_count;
    const float inv_w = (float)(1.0 / bin_width);
    const float c = (float)(1.0 / (double)inv_w);
    const float scale = (float)(32768.0 / (double)c * (1.0 - 1.0 / 256));
    char* misc = base + kJobBytes;
    unsigned long long* counters = reinterpret_cast<unsigned long long*>(misc);       // [0], [1]
    unsigned long long* overflow = counters + 2;
    float* wscale = reinterpret_cast<float*>(counters + 3);
    double* self = reinterpret_cast<double*>(counters + 4);                            // [0] atoms, [1] waters
    int32_t* dmaxbin = max_bin_out;
    char* slots = misc + kMiscBytes;
    auto cnt = [&](int k) { return reinterpret_cast<unsigned long long*>(slots + k * kSlotBytes); };
    auto dsm = [&](int k) { return reinterpret_cast<unsigned long long*>(slots + k * kSlotBytes) + kNoAllocMaxBins; };
    auto wsm = [&](int k) { return reinterpret_cast<long long*>(slots + k * kSlotBytes) + 2 * kNoAllocMaxBins; };

    // jobs of HistogramManagerMT (aa self, waters-outer x atoms-inner cross, ww self), one launch
    const float4* A = reinterpret_cast<const float4*>(atoms);
    const float4* W = reinterpret_cast<const float4*>(waters);
    struct Spec {
        const float4* a;
        int na;
        const float4* b;
        int nbp;
        int self;
    } spec[3] = {{A, n_atoms, A, n_atoms, 1}, {W, n_waters, A, n_atoms, 0}, {W, n_waters, W, n_waters, 1}};
    NoAllocInit init{};
    long long tiles_total = 0;
    auto nt = [](int n) { return (n + kNoAllocTile - 1) / kNoAllocTile; };
    for (int k = 0; k < 3; ++k) {
        const Spec& sp = spec[k];
        long long pairs = sp.self ? (long long)sp.na * (sp.na - 1) / 2 : (long long)sp.na * sp.nbp;
        if (pairs <= 0) continue;
        long long tiles = sp.self ? (long long)nt(sp.na) * (nt(sp.na) + 1) / 2 : (long long)nt(sp.na) * nt(sp.nbp);
        PairJob& J = init.jobs[init.n_jobs++];
        J.A = sp.a;
        J.B = sp.b;
        J.na = sp.na;
        J.nb = sp.nbp;
        J.self = sp.self;
        J.row_mode = kRowSingle;
        J.mult = 1;
        J.types = 0;
        J.row_lo = 0;
        J.row_hi = 1;
        J.nbins = nb;
        J.tiles_i = nt(sp.na);
        J.tiles_j = nt(sp.nbp);
        J.tile_begin = tiles_total;
        J.tile_count = tiles;
        J.inv_w = inv_w;
        J.c = c;
        J.scale = scale;
        J.counts = cnt(k);
        J.dsum = weighted_bins ? dsm(k) : nullptr;
        J.wsum = wsm(k);
        J.a_base = 0;
        J.b_base = 0;
        J.tail_end = sp.nbp;
        J.tail_from_outer = sp.self;
        tiles_total += tiles;
    }
    init.clear_words = (kMiscBytes + 3 * kSlotBytes) / 8;
    cudaError_t e = cudaSuccess;
    noalloc_init_kernel<<<64, 256, 0, s>>>(init);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
    if ((e = cudaMemsetAsync(dmaxbin, 0, sizeof(int32_t), s)) != cudaSuccess)
        return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
    weight_scale_launch(A, n_atoms, W, n_waters, wscale, s);
    weight_square_sum_launch(A, n_atoms, self, s);
    weight_square_sum_launch(W, n_waters, self + 1, s);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
    if (init.n_jobs > 0) {
        PairLaunch L{};
        L.jobs = reinterpret_cast<const PairJob*>(base);
        L.n_jobs = init.n_jobs;
        L.total_tiles = tiles_total;
        L.smem_rows = 1;
        L.smem_bins = nb;
        L.tile_counter = counters;
        L.overflow = overflow;
        L.weighted = 1;
        L.dreg = 0;
        L.wscale = wscale;
        const size_t smem = pairhist_smem_bytes(1, nb, true, kNoAllocTile);
        int sms = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess || sms <= 0)
            return fail(AUSAXS_ERR_CUDA, "cannot query the multiprocessor count");
        const int per_sm = pairhist_ctas_per_sm(smem, kNoAllocTile, false, true);
        const int grid = (int)std::min<long long>((long long)sms * per_sm, std::max<long long>(1, tiles_total));
        L.chunk = (int)std::max<long long>(1, std::min<long long>(8, tiles_total / ((long long)grid * 8)));
        pairhist_launch(L, kNoAllocTile, grid, smem, s);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
    }
    FinalizeMT F{};
    F.nb = nb;
    F.c_aa = cnt(0);
    F.c_aw = cnt(1);
    F.c_ww = cnt(2);
    F.ds_aa = dsm(0);
    F.ds_aw = dsm(1);
    F.ds_ww = dsm(2);
    F.w_aa = wsm(0);
    F.w_aw = wsm(1);
    F.w_ww = wsm(2);
    F.wscale = wscale;
    F.self_aa = self;
    F.self_ww = self + 1;
    F.bin_width = bin_width;
    F.c = c;
    F.scale = scale;
    F.weighted = weighted_bins ? 1 : 0;
    F.max_bin = dmaxbin;
    F.H = hist_out;                      // rows 0..2: aa, aw, ww
    F.tot = hist_out + 3 * (size_t)nb;   // row 3
    F.d_axis = hist_out + 4 * (size_t)nb;  // row 4
    mt_finalize_launch(F, s);
    if (overflow_out) noalloc_copy_u64<<<1, 1, 0, s>>>(overflow, overflow_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(AUSAXS_ERR_CUDA, cudaGetErrorString(e));
    return AUSAXS_OK;
}
