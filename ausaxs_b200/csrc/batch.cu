// Batched profiles: many independent structures through one persistent pair launch per tile/row
// class, one batched finalisation and one batched FP64 transform, captured once as a CUDA graph
// and replayed per call.
//
// The reference evaluates one structure per calculate_all() call
// (source/core/hist/histogram_manager/HistogramManagerMTFFAvg.cpp:194-372); a batch here is the
// same computation for n structures whose pair tiles share the GPU: every structure keeps its own
// plan (accumulators, finalisation descriptors, Debye rows) and the batch concatenates their pair
// jobs, largest structures first, into launch classes.  Tile shapes and class grouping are chosen
// by timing candidates on the batch itself (autotune) and cached per batch shape.
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

#include "engine.cuh"
#include "guard.cuh"

namespace ausaxs_b200 {
namespace {

// Pair-plan candidates of the autotuner: tile of small structures, tile of large ones, the point
// count from which a structure is large, and whether jobs are split into row classes.
struct Candidate {
    int tile_small, tile_large, threshold, by_class;
};
constexpr Candidate kCandidates[] = {
    {256, 256, 0, 0}, {256, 256, 0, 1}, {512, 512, 0, 0}, {512, 512, 0, 1},
    {256, 512, 8192, 0}, {256, 512, 8192, 1}, {256, 512, 24576, 1},
};
constexpr int kNumCandidates = sizeof(kCandidates) / sizeof(kCandidates[0]);
constexpr int kDefaultCandidate = 5;

// choice per batch shape (structures, pairs, bins, SMs), shared by all batches of the process
std::mutex g_tune_mutex;
std::map<std::tuple<int, long long, int, int>, int> g_tuned;

// One structure's destinations for new coordinates (ausaxs_gpu_batch_set_points): its atoms are rows
// [a0, a0 + na) of the concatenated input, its waters rows [w0, w0 + nw).
struct PointsItem {
    long long a0, na, w0, nw;
    float4* raw_a;
    float4* dense_a;
    float4* raw_w;
};

__device__ __forceinline__ bool finite3(const float4& v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

// New x, y, z for every point of every structure (block row y: structure y, y + gridDim.y, ...).  An
// atom keeps its form-factor type: one whose input type differs from it, or a point with a
// non-finite coordinate, is left as it was and counted in *rejected, so the per-type counts of the
// plans (and the type rows the pair kernel indexes) always hold.
__global__ void set_points_kernel(const PointsItem* items, int n, const float4* atoms, const float4* waters,
                                  unsigned long long* rejected) {
    unsigned int bad = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int s = blockIdx.y; s < n; s += gridDim.y) {
        const PointsItem it = items[s];
        for (long long k = first; k < it.na; k += stride) {
            const float4 v = atoms[it.a0 + k];
            const float4 old = it.raw_a[k];
            if (__float_as_int(v.w) != __float_as_int(old.w) || !finite3(v)) {
                ++bad;
                continue;
            }
            it.raw_a[k] = v;
            const float dense_type = it.dense_a[k].w;
            it.dense_a[k] = make_float4(v.x, v.y, v.z, dense_type);
        }
        for (long long k = first; k < it.nw; k += stride) {
            const float4 v = waters[it.w0 + k];
            if (!finite3(v)) {
                ++bad;
                continue;
            }
            it.raw_w[k] = make_float4(v.x, v.y, v.z, it.raw_w[k].w);
        }
    }
    if (bad) atomicAdd(rejected, (unsigned long long)bad);
}

}  // namespace

struct Batch {
    Ctx* ctx = nullptr;
    ausaxs_hist_config cfg{};
    std::vector<std::unique_ptr<Structure>> items;
    std::vector<ausaxs_hist_config> cfgs;  // per structure (z_exv)
    std::vector<int> order;                // structures by pair count, largest first
    int max_nb = 0;
    long long pairs = 0;
    struct Launch {
        PairLaunch L{};
        int tile = 256, grid = 0;
        size_t smem = 0;
    };
    std::vector<Launch> launches;
    int choice = -1;
    // misc: tile counters [0, 16), overflow [16] (set from [24] at the start of every profile), q values
    // recomputed in FP64 [20], points rejected by the last set_points [24] (kept across profiles)
    DevBuf jobs, misc, zero, fin, args;
    DevBuf qfactors;      // the per-q factor table every structure's transform reads
    DebyeArgs qf_args{};  // q and parameters of the table
    std::vector<long long> a_off, w_off;  // creation offsets of the concatenated atoms and waters
    DevBuf points_items, points_in;       // set_points: destinations, staged host input
    // exact-accumulation tensor-core transform (debye_x.cu): Taylor tables shared by every structure,
    // left-operand rows of all structures (largest first), per-structure partial sums and bound terms
    struct XState {
        bool on = false;
        XPlan plan{};
        DevBuf table, cpart, rows, planes, flags, qcache, adig, tile_off, row_scale;
    } x;
    DevBuf d_stats;                      // census of every structure (creation only)
    DevBuf arena;                        // every structure's point arrays
    PrepStats* h_stats = nullptr;        // pinned slots owned by the context
    int n_zero = 0;
    cudaStream_t side[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
    // recorded around the pair stage inside the captured profile: the pair launches' device time of
    // the last replay (ausaxs_gpu_batch_pair_time)
    cudaEvent_t pair_t0 = nullptr, pair_t1 = nullptr;
    // captured profile
    cudaGraphExec_t exec = nullptr;
    long long graph_launches = 0;
    struct Key {
        const double* q = nullptr;
        int nq = -1;
        double* I = nullptr;
        int choice = -1;
        cudaStream_t s = nullptr;
        ausaxs_debye_params p{};
    } key;

    ~Batch() {
        if (ctx && ctx->stream) cudaStreamSynchronize(ctx->stream);
        if (exec) cudaGraphExecDestroy(exec);
        for (auto& st : side)
            if (st) cudaStreamDestroy(st);
        if (fork) cudaEventDestroy(fork);
        for (auto& e : join)
            if (e) cudaEventDestroy(e);
        if (pair_t0) cudaEventDestroy(pair_t0);
        if (pair_t1) cudaEventDestroy(pair_t1);
    }

    unsigned long long* overflow() const { return misc.as<unsigned long long>() + 16; }
    unsigned long long* rejected() const { return misc.as<unsigned long long>() + 24; }
    // q values of the last profile that the FP64 transform recomputed (cleared by every replay)
    int32_t* fp64_count() const { return reinterpret_cast<int32_t*>(misc.as<unsigned long long>() + 20); }

    void load(const ausaxs_hist_config& c, int n, const float* atoms, const int64_t* aoff, const float* waters,
              const int64_t* woff, const float* exv, const int64_t* xoff, const double* z_exv, bool host) {
        if (c.manager != AUSAXS_MANAGER_FFAVG && c.manager != AUSAXS_MANAGER_FFGRID)
            throw Error{AUSAXS_ERR_ARGUMENT, "batched profiles support the FFAVG and FFGRID managers"};
        if (n <= 0 || !aoff || !woff) throw Error{AUSAXS_ERR_ARGUMENT, "empty batch or missing offsets"};
        const bool grid = c.manager == AUSAXS_MANAGER_FFGRID;
        if (grid && !xoff) throw Error{AUSAXS_ERR_ARGUMENT, "FFGRID batches need excluded-volume offsets"};
        cfg = c;
        // every structure's copies and census first, one synchronisation, then validation and plans
        h_stats = ctx->stats_slots(n);
        d_stats.ensure(sizeof(PrepStats) * n);
        // one arena for every structure's point arrays (raw atoms, waters, dummies, dense atoms, type
        // table) instead of five allocations per structure
        auto pts = [](int64_t k) { return align_up((size_t)std::max<int64_t>(1, k) * 16, 256); };
        size_t arena_bytes = 0;
        for (int i = 0; i < n; ++i) {
            const int64_t na = aoff[i + 1] - aoff[i], nw = woff[i + 1] - woff[i];
            const int64_t nx = grid ? xoff[i + 1] - xoff[i] : 0;
            if (na < 0 || nw < 0 || nx < 0 || na > INT32_MAX || nw > INT32_MAX || nx > INT32_MAX)
                throw Error{AUSAXS_ERR_ARGUMENT, "bad offsets"};
            arena_bytes += 2 * pts(na) + pts(nw) + pts(nx) + 256;
        }
        arena.ensure(arena_bytes);
        a_off.assign(aoff, aoff + n + 1);
        w_off.assign(woff, woff + n + 1);
        size_t at = 0;
        for (int i = 0; i < n; ++i) {
            const int64_t na = aoff[i + 1] - aoff[i], nw = woff[i + 1] - woff[i];
            const int64_t nx = grid ? xoff[i + 1] - xoff[i] : 0;
            auto S = std::make_unique<Structure>();
            S->ctx = ctx;
            auto take = [&](DevBuf& b, size_t bytes) {
                b.view(arena.as<char>(at), bytes);
                at += bytes;
            };
            take(S->raw_a, pts(na));
            take(S->dense_a, pts(na));
            take(S->raw_w, pts(nw));
            take(S->raw_x, pts(nx));
            take(S->meta, 256);
            S->load_begin(atoms ? atoms + 4 * aoff[i] : nullptr, (int)na, waters ? waters + 4 * woff[i] : nullptr,
                          (int)nw, grid && exv ? exv + 4 * xoff[i] : nullptr, (int)nx, 1, host, h_stats + i,
                          d_stats.as<PrepStats>() + i);
            items.push_back(std::move(S));
        }
        AUSAXS_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int i = 0; i < n; ++i) {
            Structure& S = *items[i];
            S.load_end(h_stats[i]);
            ausaxs_hist_config ci = c;
            if (z_exv) ci.z_exv = z_exv[i];
            S.plan_for(ci);
            max_nb = std::max(max_nb, S.plan.nb);
            pairs += S.plan.pairs;
            cfgs.push_back(ci);
        }
        order.resize(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(),
                         [&](int a, int b) { return items[a]->plan.pairs > items[b]->plan.pairs; });
        // accumulators to clear before each run (one range per structure) and the batch counters
        std::vector<ZeroRange> zr;
        for (auto& S : items) {
            Plan& P = S->plan;
            zr.push_back({P.dev.as<unsigned long long>(P.off_acc), (long long)(P.acc_bytes / 8)});
        }
        misc.ensure(256);
        AUSAXS_CUDA(cudaMemset(misc.p, 0, 256));
        zr.push_back({misc.as<unsigned long long>(), 16});
        zr.push_back({overflow(), 1, rejected()});  // rejected points poison every profile until replaced
        zr.push_back({overflow() + 1, 7});
        n_zero = (int)zr.size();
        zero.ensure(sizeof(ZeroRange) * zr.size());
        AUSAXS_CUDA(cudaMemcpy(zero.p, zr.data(), sizeof(ZeroRange) * zr.size(), cudaMemcpyHostToDevice));
        std::vector<FinalizeFF> fins;
        for (auto& S : items) fins.push_back(S->plan.fin_ff);
        fin.ensure(sizeof(FinalizeFF) * fins.size());
        AUSAXS_CUDA(cudaMemcpy(fin.p, fins.data(), sizeof(FinalizeFF) * fins.size(), cudaMemcpyHostToDevice));
        for (auto& st : side) AUSAXS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        AUSAXS_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
        for (auto& e : join) AUSAXS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        AUSAXS_CUDA(cudaEventCreate(&pair_t0));
        AUSAXS_CUDA(cudaEventCreate(&pair_t1));
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        auto it = g_tuned.find(shape());
        build(it != g_tuned.end() ? it->second : kDefaultCandidate);
    }

    std::tuple<int, long long, int, int> shape() const { return {(int)items.size(), pairs, max_nb, ctx->sm_count}; }

    // job tables and launch shapes of one candidate
    void build(int c_idx) {
        const Candidate& c = kCandidates[c_idx];
        std::vector<PairJob> js[2][3];
        long long tiles[2][3] = {{0, 0, 0}, {0, 0, 0}};
        int rows[2][3] = {{1, 1, 1}, {1, 1, 1}};
        const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
        // on-chip rows that fit next to the batch-wide bin count
        if (pairhist_launch_smem(1, max_nb, false, 512) > kPairSmemCap)
            throw Error{AUSAXS_ERR_CAPACITY, "too many distance bins for a batched launch"};
        const int max_rows = pairhist_max_rows(max_nb, false);
        for (int i : order) {
            const Structure& S = *items[i];
            const int biggest = std::max({S.n_a, S.n_w, grid ? S.n_x : 0});
            const int b = (c.tile_small != c.tile_large && biggest >= c.threshold) ? 1 : 0;
            append_pair_jobs(S.plan, b ? c.tile_large : c.tile_small, c.by_class != 0, js[b], tiles[b], rows[b], max_rows);
        }
        size_t n_jobs = 0;
        for (auto& bb : js)
            for (auto& g : bb) n_jobs += g.size();
        if (exec) {
            cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
        jobs.ensure(sizeof(PairJob) * std::max<size_t>(1, n_jobs));
        launches.clear();
        size_t at = 0;
        int counter = 0;
        for (int b = 0; b < 2; ++b)
            for (int g = 0; g < 3; ++g) {
                if (js[b][g].empty()) continue;
                Launch La;
                La.tile = b ? c.tile_large : c.tile_small;
                La.smem = pairhist_launch_smem(rows[b][g], max_nb, false, La.tile);
                if (La.smem > kPairSmemCap) throw Error{AUSAXS_ERR_CAPACITY, "too many distance bins for a batched launch"};
                const int per_sm =
                    pairhist_ctas_per_sm(La.smem, La.tile, pairhist_dreg(rows[b][g], max_nb, false, La.tile), false);
                La.grid = (int)std::min<long long>((long long)ctx->sm_count * per_sm, std::max<long long>(1, tiles[b][g]));
                PairLaunch& L = La.L;
                L.jobs = jobs.as<PairJob>() + at;
                L.n_jobs = (int)js[b][g].size();
                L.total_tiles = tiles[b][g];
                L.chunk = (int)std::max<long long>(1, std::min<long long>(8, tiles[b][g] / ((long long)La.grid * 8)));
                L.smem_rows = rows[b][g];
                L.smem_bins = max_nb;
                L.tile_counter = misc.as<unsigned long long>() + counter++;
                L.overflow = overflow();
                L.weighted = 0;
                L.dreg = pairhist_dreg(rows[b][g], max_nb, false, La.tile) ? 1 : 0;
                L.wscale = nullptr;
                L.inv_w = items.empty() ? 0.f : items[order[0]]->plan.inv_w;
                AUSAXS_CUDA(cudaMemcpy(jobs.as<PairJob>() + at, js[b][g].data(), sizeof(PairJob) * js[b][g].size(),
                                       cudaMemcpyHostToDevice));
                at += js[b][g].size();
                launches.push_back(La);
            }
        choice = c_idx;
    }

    // clear the accumulators, then the pair launches: the first on s, the others forked onto the
    // side streams so a class's tail overlaps the next class
    void enqueue_pairs(cudaStream_t s) {
        Ctx& C = *ctx;
        zero_ranges_launch(zero.as<ZeroRange>(), n_zero, s);
        C.check_launch("zero");
        const int n = (int)launches.size();
        if (n > 1) AUSAXS_CUDA(cudaEventRecord(fork, s));
        for (int k = 0; k < n; ++k) {
            cudaStream_t sk = k == 0 ? s : side[(k - 1) % 2];
            if (k > 0 && k <= 2) AUSAXS_CUDA(cudaStreamWaitEvent(sk, fork, 0));
            const Launch& La = launches[k];
            pairhist_launch(La.L, La.tile, La.grid, La.smem, sk);
            C.check_launch("pairhist");
        }
        for (int k = 1; k <= std::min(2, n - 1); ++k) {
            AUSAXS_CUDA(cudaEventRecord(join[k - 1], side[k - 1]));
            AUSAXS_CUDA(cudaStreamWaitEvent(s, join[k - 1], 0));
        }
    }

    // the tensor-core stage's tables, rows and partial-sum planes for q (device, nq values), and the
    // fields of every structure's transform arguments that point at them
    void setup_x(const double* q, int nq, std::vector<DebyeArgs>& A) {
        std::vector<double> hq(nq);
        AUSAXS_CUDA(cudaMemcpy(hq.data(), q, sizeof(double) * nq, cudaMemcpyDeviceToHost));
        double qmax = 0;
        for (double v : hq) qmax = std::max(qmax, std::fabs(v));
        XState& X = x;
        XPlan& XP = X.plan;
        XP.w = cfg.bin_width;
        XP.nq = nq;
        XP.K = debye_x_order(qmax, XP.w);
        XP.nch = std::max(1, (max_nb + kXChunk - 1) / kXChunk);
        // splits of the chunk range: at most debye_x_max_chunks per split (exact s32 sums), and
        // enough of them for two CTAs per SM
        long long n_rows = 0;
        for (auto& S : items) n_rows += S->plan.R;
        const long long tiles = (long long)((nq + kXQTile - 1) / kXQTile) * ((n_rows + 127) / 128);
        int splits = (XP.nch + debye_x_max_chunks(XP.K) - 1) / debye_x_max_chunks(XP.K);
        while (splits < XP.nch && tiles * splits < 2LL * ctx->sm_count) ++splits;
        XP.cps = (XP.nch + splits - 1) / splits;
        XP.splits = (XP.nch + XP.cps - 1) / XP.cps;
        X.table.ensure(debye_x_table_bytes(nq, XP.nch, XP.K));
        const size_t ncp = debye_x_cpart_doubles(nq, XP.nch);
        X.cpart.ensure(sizeof(double) * ncp);
        const int nqp = (int)(ncp / XP.nch);
        X.qcache.ensure(sizeof(double) * nq);
        AUSAXS_CUDA(cudaMemset(X.qcache.p, 0xff, sizeof(double) * nq));  // NaN: the tables are made on first use
        X.flags.ensure(256);
        AUSAXS_CUDA(cudaMemset(X.flags.p, 0, 256));
        // per structure: values [splits][R][nq], then e1, e0, habs [splits][R]
        std::vector<size_t> at(items.size());
        size_t total = 0;
        for (size_t i = 0; i < items.size(); ++i) {
            at[i] = total;
            const size_t R = items[i]->plan.R;
            total += align_up((size_t)XP.splits * R * nq + 3 * (size_t)XP.splits * R, 32);
        }
        X.planes.ensure(sizeof(double) * std::max<size_t>(1, total));
        double* base = X.planes.as<double>();
        std::vector<XRow> rows;
        std::vector<int> row_chunks;  // chunk bound of each row (its plan's bins)
        for (int i : order) {
            Structure& S = *items[i];
            Plan& P = S.plan;
            const int R = P.R;
            char* pb = P.dev.as<char>();
            double* v = base + at[i];
            double* e1 = v + (size_t)XP.splits * R * nq;
            double* e0 = e1 + (size_t)XP.splits * R;
            double* ha = e0 + (size_t)XP.splits * R;
            const double* axes[3] = {reinterpret_cast<const double*>(pb + P.off_d),
                                     reinterpret_cast<const double*>(pb + P.off_dax),
                                     reinterpret_cast<const double*>(pb + P.off_dxx)};
            const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
            for (int r = 0; r < R; ++r) {
                const int g = grid ? P.rows_host[r].group : 0;
                XRow xr{};
                xr.H = reinterpret_cast<const double*>(pb + P.off_H) + (size_t)r * P.nb;
                xr.axis = axes[g];
                xr.max_bin = reinterpret_cast<const int32_t*>(pb + P.off_maxbin);
                xr.out = v + (size_t)r * nq;
                xr.e1 = e1 + r;
                xr.e0 = e0 + r;
                xr.habs = ha + r;
                xr.out_z = (long long)R * nq;
                xr.e_z = R;
                rows.push_back(xr);
                row_chunks.push_back((P.nb + kXChunk - 1) / kXChunk);
            }
            DebyeArgs& a = A[i];
            a.x_v = v;
            a.x_e1 = e1;
            a.x_e0 = e0;
            a.x_habs = ha;
            a.x_splits = XP.splits;
            a.x_cpart = X.cpart.as<double>();
            a.x_nch = XP.nch;
            a.x_nqp = nqp;
            a.x_K = XP.K;
            a.x_ctr = debye_x_trunc(XP.K, XP.w);
            a.tc_error = X.flags.as<int32_t>() + 1;
        }
        XP.n_rows = (int)rows.size();
        X.rows.ensure(sizeof(XRow) * std::max<size_t>(1, rows.size()));
        AUSAXS_CUDA(cudaMemcpy(X.rows.p, rows.data(), sizeof(XRow) * rows.size(), cudaMemcpyHostToDevice));
        // the rows' digit blocks: per M tile, its rows' largest chunk bound (capped by the table's)
        const int n_tiles = (XP.n_rows + 127) / 128;
        std::vector<long long> toff(n_tiles);
        long long adig = 0;
        for (int t = 0; t < n_tiles; ++t) {
            int ch = 0;
            for (int r = t * 128; r < std::min(XP.n_rows, (t + 1) * 128); ++r) ch = std::max(ch, row_chunks[r]);
            toff[t] = adig;
            adig += (long long)std::min(ch, XP.nch) * XP.K * (long long)debye_x_block_bytes();
        }
        X.adig.ensure((size_t)std::max<long long>(256, adig));
        X.tile_off.ensure(sizeof(long long) * n_tiles);
        AUSAXS_CUDA(cudaMemcpy(X.tile_off.p, toff.data(), sizeof(long long) * n_tiles, cudaMemcpyHostToDevice));
        X.row_scale.ensure(sizeof(double) * XP.n_rows);
        XP.rows = X.rows.as<XRow>();
        XP.table = X.table.as<unsigned char>();
        XP.cpart = X.cpart.as<double>();
        XP.q_cached = X.qcache.as<double>();
        XP.flags = X.flags.as<int32_t>();
        XP.adig = X.adig.as<unsigned char>();
        XP.tile_off = X.tile_off.as<long long>();
        XP.row_scale = X.row_scale.as<double>();
        X.on = true;
    }

    void enqueue_all(const double* q, int nq, cudaStream_t s) {
        // external records: event-record nodes of the captured graph (a plain record in a capture only
        // orders streams), so every replay timestamps the pair stage
        AUSAXS_CUDA(cudaEventRecordWithFlags(pair_t0, s, cudaEventRecordExternal));
        enqueue_pairs(s);
        AUSAXS_CUDA(cudaEventRecordWithFlags(pair_t1, s, cudaEventRecordExternal));
        ff_finalize_batch_launch(fin.as<FinalizeFF>(), (int)items.size(), max_nb, s);
        ctx->check_launch("finalize");
        ctx->launches += 1;  // two kernels
        if (x.on) {
            if (!debye_x_enqueue(x.plan, q, s)) throw Error{AUSAXS_ERR_CUDA, "cannot launch the tensor-core Debye transform"};
            ctx->check_launch("debye_x");
            ctx->launches += 4;  // five kernels
        }
        // every structure shares q, the parameters and the excluded-volume model: one factor table
        debye_qfactors_launch(qf_args, qfactors.as<double>(), s);
        ctx->check_launch("qfactors");
        int max_R = 1;
        for (auto& S : items) max_R = std::max(max_R, S->plan.R);
        debye_fp64_batch_launch(args.as<DebyeArgs>(), (int)items.size(), nq, max_R, s);
        ctx->check_launch("debye");
    }

    // I[i * nq + k] for every structure i (FP64 transform for every q); replays the captured graph
    void profile_device(const double* q, int nq, const ausaxs_debye_params& p, double* I) {
        Ctx& C = *ctx;
        cudaStream_t s = C.stream;
        const ausaxs_debye_params& o = key.p;
        const bool same_p = o.cw == p.cw && o.cx == p.cx && o.crho == p.crho && o.dw_atomic == p.dw_atomic &&
                            o.dw_exv == p.dw_exv && o.grid_width == p.grid_width && o.precision == p.precision &&
                            o.tolerance == p.tolerance;
        const bool same = exec && key.q == q && key.nq == nq && key.I == I && key.choice == choice && key.s == s && same_p;
        if (!same) {
            if (exec) {
                cudaGraphExecDestroy(exec);
                exec = nullptr;
            }
            std::vector<DebyeArgs> A;
            for (size_t i = 0; i < items.size(); ++i) {
                DebyeArgs a = items[i]->debye_args(cfgs[i], q, nq, p, I + i * (size_t)nq, nullptr);
                a.overflow = overflow();  // the batch's launches share one overflow counter
                a.fp64_columns = fp64_count();
                A.push_back(a);
            }
            x.on = false;
            if (p.precision != 1) setup_x(q, nq, A);
            qfactors.ensure(sizeof(double) * debye_qfactors_doubles(nq));
            qf_args = A[0];
            for (auto& a : A) a.qf = qfactors.as<double>();
            args.ensure(sizeof(DebyeArgs) * A.size());
            AUSAXS_CUDA(cudaMemcpyAsync(args.p, A.data(), sizeof(DebyeArgs) * A.size(), cudaMemcpyHostToDevice, s));
            AUSAXS_CUDA(cudaStreamSynchronize(s));
            cudaGraph_t g = nullptr;
            AUSAXS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            const long long launches0 = C.launches;
            try {
                enqueue_all(q, nq, s);
            } catch (...) {
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            AUSAXS_CUDA(cudaStreamEndCapture(s, &g));
            graph_launches = C.launches - launches0;  // kernels per replay (counted as they were captured)
            C.launches = launches0;
            cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                exec = nullptr;
                throw Error{AUSAXS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e)};
            }
            key.q = q;
            key.nq = nq;
            key.I = I;
            key.choice = choice;
            key.s = s;
            key.p = p;
        }
        AUSAXS_CUDA(cudaGraphLaunch(exec, s));
        C.launches += graph_launches;
    }

    // New coordinates for every point, in the creation layout (rows aoff[i] .. aoff[i+1] of atoms,
    // woff[i] .. woff[i+1] of waters), with every atom's form-factor type as at creation.  The plans,
    // job tables and captured graph stay: bins were planned from the creation coordinates, so pairs
    // that now lie beyond them show as bin overflow in the next profile.  Host input is staged with
    // one copy per array; host calls synchronise and report rejected points.
    // z_exv (host, may be null: kept) replaces the structures' excluded-volume charges per atom.
    void set_points(const float* atoms, const float* waters, const double* z_exv, bool host) {
        if (cfg.manager != AUSAXS_MANAGER_FFAVG)
            throw Error{AUSAXS_ERR_ARGUMENT, "new coordinates need an FFAVG batch (FFGRID dummies follow the atoms)"};
        Ctx& C = *ctx;
        cudaStream_t s = C.stream;
        const int n = (int)items.size();
        const long long na = a_off[n] - a_off[0], nw = w_off[n] - w_off[0];
        if ((na && !atoms) || (nw && !waters)) throw Error{AUSAXS_ERR_ARGUMENT, "null point array"};
        if (!points_items.p) {
            std::vector<PointsItem> v(n);
            for (int i = 0; i < n; ++i) {
                Structure& S = *items[i];
                v[i] = {a_off[i] - a_off[0], S.n_a, w_off[i] - w_off[0], S.n_w,
                        S.raw_a.as<float4>(), S.dense_a.as<float4>(), S.raw_w.as<float4>()};
            }
            points_items.ensure(sizeof(PointsItem) * n);
            AUSAXS_CUDA(cudaMemcpy(points_items.p, v.data(), sizeof(PointsItem) * n, cudaMemcpyHostToDevice));
        }
        const float4* src_a = reinterpret_cast<const float4*>(atoms) + a_off[0];
        const float4* src_w = reinterpret_cast<const float4*>(waters) + w_off[0];
        if (host) {
            points_in.ensure((size_t)std::max<long long>(1, na + nw) * 16);
            float4* in = points_in.as<float4>();
            if (na) AUSAXS_CUDA(cudaMemcpyAsync(in, src_a, (size_t)na * 16, cudaMemcpyHostToDevice, s));
            if (nw) AUSAXS_CUDA(cudaMemcpyAsync(in + na, src_w, (size_t)nw * 16, cudaMemcpyHostToDevice, s));
            src_a = in;
            src_w = in + na;
        }
        if (z_exv) {
            std::vector<FinalizeFF> fins;
            for (int i = 0; i < n; ++i) {
                if (!std::isfinite(z_exv[i])) throw Error{AUSAXS_ERR_ARGUMENT, "non-finite z_exv"};
                cfgs[i].z_exv = z_exv[i];
                items[i]->plan.fin_ff.z_exv = z_exv[i];
                fins.push_back(items[i]->plan.fin_ff);
            }
            // pageable source: staged before the call returns, ordered after earlier replays on s
            AUSAXS_CUDA(cudaMemcpyAsync(fin.p, fins.data(), sizeof(FinalizeFF) * n, cudaMemcpyHostToDevice, s));
        }
        AUSAXS_CUDA(cudaMemsetAsync(rejected(), 0, 8, s));
        long long most = 1;
        for (auto& S : items) most = std::max<long long>({most, (long long)S->n_a, (long long)S->n_w});
        const dim3 grid((unsigned)std::min<long long>(64, (most + 1023) / 1024), (unsigned)std::min(n, 65535));
        set_points_kernel<<<grid, 256, 0, s>>>(points_items.as<PointsItem>(), n, src_a, src_w, rejected());
        C.check_launch("set_points");
        if (host) {
            unsigned long long bad = 0;
            AUSAXS_CUDA(cudaMemcpyAsync(&bad, rejected(), 8, cudaMemcpyDeviceToHost, s));
            AUSAXS_CUDA(cudaStreamSynchronize(s));
            if (bad)
                throw Error{AUSAXS_ERR_ARGUMENT, std::to_string(bad) +
                                                     " points rejected: a form-factor type differs from the batch's or a "
                                                     "coordinate is not finite"};
        }
    }

    // times every candidate's pair launches on this batch (best of 2 after a warm-up) and keeps the fastest
    int autotune(double* times_ms, int n_times) {
        Ctx& C = *ctx;
        cudaStream_t s = C.stream;
        cudaEvent_t e0, e1;
        AUSAXS_CUDA(cudaEventCreate(&e0));
        AUSAXS_CUDA(cudaEventCreate(&e1));
        int best = -1;
        float best_ms = 0;
        for (int c = 0; c < kNumCandidates; ++c) {
            build(c);
            enqueue_pairs(s);
            float ms = 1e30f;
            for (int rep = 0; rep < 2; ++rep) {
                AUSAXS_CUDA(cudaEventRecord(e0, s));
                enqueue_pairs(s);
                AUSAXS_CUDA(cudaEventRecord(e1, s));
                AUSAXS_CUDA(cudaEventSynchronize(e1));
                float t = 0;
                AUSAXS_CUDA(cudaEventElapsedTime(&t, e0, e1));
                ms = std::min(ms, t);
            }
            if (times_ms && c < n_times) times_ms[c] = ms;
            if (best < 0 || ms < best_ms) {
                best = c;
                best_ms = ms;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        build(best);
        std::lock_guard<std::mutex> lk(g_tune_mutex);
        g_tuned[shape()] = best;
        return best;
    }
};

}  // namespace ausaxs_b200

using namespace ausaxs_b200;

struct ausaxs_gpu_batch {
    Batch impl;
};

extern "C" {

int ausaxs_gpu_batch_create(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, int32_t n_structures,
                            const float* atoms, const int64_t* atom_offsets, const float* waters,
                            const int64_t* water_offsets, const float* exv, const int64_t* exv_offsets,
                            const double* z_exv, int32_t host_pointers, ausaxs_gpu_batch** out) {
    return guarded([&] {
        if (!ctx || !cfg || !out) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        *out = nullptr;
        AUSAXS_CUDA(cudaSetDevice(ctx->impl.device));
        auto* b = new ausaxs_gpu_batch();
        b->impl.ctx = &ctx->impl;
        try {
            b->impl.load(*cfg, n_structures, atoms, atom_offsets, waters, water_offsets, exv, exv_offsets, z_exv,
                         host_pointers != 0);
        } catch (...) {
            delete b;
            throw;
        }
        *out = b;
    });
}

int ausaxs_gpu_batch_destroy(ausaxs_gpu_batch* b) {
    return guarded([&] {
        if (!b) return;
        cudaStreamSynchronize(b->impl.ctx->stream);
        delete b;
    });
}

int ausaxs_gpu_batch_autotune(ausaxs_gpu_batch* b, int32_t* choice, double* times_ms, int32_t n_times) {
    return guarded([&] {
        if (!b) throw Error{AUSAXS_ERR_ARGUMENT, "null batch"};
        AUSAXS_CUDA(cudaSetDevice(b->impl.ctx->device));
        const int c = b->impl.autotune(times_ms, n_times);
        if (choice) *choice = c;
    });
}

int ausaxs_gpu_batch_candidate(int32_t index, int32_t* tile_small, int32_t* tile_large, int32_t* threshold,
                               int32_t* by_class) {
    return guarded([&] {
        if (index < 0 || index >= kNumCandidates) throw Error{AUSAXS_ERR_ARGUMENT, "no such candidate"};
        const Candidate& c = kCandidates[index];
        if (tile_small) *tile_small = c.tile_small;
        if (tile_large) *tile_large = c.tile_large;
        if (threshold) *threshold = c.threshold;
        if (by_class) *by_class = c.by_class;
    });
}

int ausaxs_gpu_batch_profile_device(ausaxs_gpu_batch* b, const double* q, int32_t n_q,
                                    const ausaxs_debye_params* params, double* Iq) {
    return guarded([&] {
        if (!b || !q || !Iq || n_q <= 0 || !params) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        AUSAXS_CUDA(cudaSetDevice(b->impl.ctx->device));
        b->impl.profile_device(q, n_q, *params, Iq);
    });
}

int ausaxs_gpu_batch_profile(ausaxs_gpu_batch* b, const double* q, int32_t n_q, const ausaxs_debye_params* params,
                             double* Iq) {
    return guarded([&] {
        if (!b || !q || !Iq || n_q <= 0 || !params) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Batch& B = b->impl;
        Ctx& C = *B.ctx;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const size_t n = B.items.size();
        const size_t bytes_q = ((size_t)n_q * 8 + 255) & ~(size_t)255;
        C.io.ensure(bytes_q + n * n_q * 8 + 256);
        double* dq = C.io.as<double>();
        double* dI = C.io.as<double>(bytes_q);
        AUSAXS_CUDA(cudaMemcpyAsync(dq, q, (size_t)n_q * 8, cudaMemcpyHostToDevice, C.stream));
        B.profile_device(dq, n_q, *params, dI);
        AUSAXS_CUDA(cudaMemcpyAsync(Iq, dI, n * n_q * 8, cudaMemcpyDeviceToHost, C.stream));
        unsigned long long flags[2] = {0, 0};
        AUSAXS_CUDA(cudaMemcpyAsync(&flags[0], B.overflow(), 8, cudaMemcpyDeviceToHost, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(&flags[1], B.rejected(), 8, cudaMemcpyDeviceToHost, C.stream));
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
        if (flags[1])
            throw Error{AUSAXS_ERR_ARGUMENT, "the last ausaxs_gpu_batch_set_points rejected points (changed form-factor "
                                             "type or non-finite coordinate)"};
        if (flags[0])
            throw Error{AUSAXS_ERR_BIN_OVERFLOW, "pair distances beyond the batch's bins (bin_count * bin_width, or the "
                                                 "range planned from the creation coordinates after set_points)"};
    });
}

int ausaxs_gpu_batch_fp64_columns(ausaxs_gpu_batch* b, int64_t* n) {
    return guarded([&] {
        if (!b || !n) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Batch& B = b->impl;
        AUSAXS_CUDA(cudaSetDevice(B.ctx->device));
        int32_t v = 0;
        AUSAXS_CUDA(cudaMemcpyAsync(&v, B.fp64_count(), sizeof(v), cudaMemcpyDeviceToHost, B.ctx->stream));
        AUSAXS_CUDA(cudaStreamSynchronize(B.ctx->stream));
        *n = v;
    });
}

int ausaxs_gpu_batch_set_points(ausaxs_gpu_batch* b, const float* atoms, const float* waters, const double* z_exv,
                                int32_t host_pointers) {
    return guarded([&] {
        if (!b) throw Error{AUSAXS_ERR_ARGUMENT, "null batch"};
        AUSAXS_CUDA(cudaSetDevice(b->impl.ctx->device));
        b->impl.set_points(atoms, waters, z_exv, host_pointers != 0);
    });
}

int ausaxs_gpu_batch_pair_time(ausaxs_gpu_batch* b, double* ms) {
    return guarded([&] {
        if (!b || !ms) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Batch& B = b->impl;
        AUSAXS_CUDA(cudaSetDevice(B.ctx->device));
        if (!B.exec) throw Error{AUSAXS_ERR_ARGUMENT, "the batch has not been profiled"};
        AUSAXS_CUDA(cudaEventSynchronize(B.pair_t1));
        float t = 0;
        AUSAXS_CUDA(cudaEventElapsedTime(&t, B.pair_t0, B.pair_t1));
        *ms = t;
    });
}

int ausaxs_gpu_batch_histogram(ausaxs_gpu_batch* b, int32_t index, ausaxs_hist_result* out) {
    return guarded([&] {
        if (!b || !out || index < 0 || index >= (int)b->impl.items.size()) throw Error{AUSAXS_ERR_ARGUMENT, "bad argument"};
        AUSAXS_CUDA(cudaSetDevice(b->impl.ctx->device));
        b->impl.items[index]->read_histogram(b->impl.cfgs[index], out);
    });
}

}  // extern "C"
