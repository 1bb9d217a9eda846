// Serving loop for rigid-body refinement: device-resident multi-body assemblies whose I(q) and
// chi-square are updated after a rigid move of one body by recomputing only the partial histograms
// between that body and the others.
//
// The reference's incremental path is PartialHistogramManagerMT (PartialHistogramManagerMT.cpp:42-170
// and :308-341): per-body self partials, per-body-pair cross partials and master = sum of partials,
// updated as master -= old + new; it exists for the Simple model only (the form-factor variants are
// disabled in HistogramSettings.h:34-36).  Here the FFAvg histograms (aa by type pair, aw by atom
// type, ww) are decomposed the same way, and a move recomputes every partial with the moved body,
// its self partials included.  Every pair job carries the full assembly's row geometry
// (PairJob a_base/b_base/tail_end), so each pair is evaluated exactly as in a full
// HistogramManagerMTFFAvg::calculate_all() of the moved assembly; all accumulation is integer, so
// the master (the sum of the partials) equals the full recompute bit for bit, whether a request runs
// alone or overlaps others.
//
// Requests of one assembly run in order; requests of different assemblies overlap on the device.  A
// server admits assemblies while their device footprint fits its memory budget and requests while an
// output slot is free (continuous batching: a request is admitted as soon as a slot frees, without
// waiting for the others in flight).  Scheduling on the device: every assembly has a high- and a
// low-priority stream; a move whose pair count is at most the median over the server's bodies goes to
// the high-priority one (an event keeps each assembly's requests in order across its two streams), and
// the pair launches of requests are made of short-lived CTAs (a few tiles each) instead of one
// persistent grid, so the block scheduler hands SMs to a small move as soon as running CTAs finish
// instead of after a large move's whole launch.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <map>
#include <thread>

#include "engine.cuh"
#include "guard.cuh"
#include "lsq.cuh"

namespace ausaxs_b200 {
namespace {

struct Pose {
    double R[9];
    double t[3];
};

// x <- R x + t in FP64 from the body's original coordinates (Body::rotate then Body::translate,
// source/core/data/Body.cpp:135-156, composed on the host), rounded to float
__global__ void transform_kernel(const float4* __restrict__ src, float4* __restrict__ dst, int n, Pose p) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = src[i];
        const double x = v.x, y = v.y, z = v.z;
        float4 o;
        o.x = static_cast<float>(p.R[0] * x + p.R[1] * y + p.R[2] * z + p.t[0]);
        o.y = static_cast<float>(p.R[3] * x + p.R[4] * y + p.R[5] * z + p.t[1]);
        o.z = static_cast<float>(p.R[6] * x + p.R[7] * y + p.R[8] * z + p.t[2]);
        o.w = v.w;
        dst[i] = o;
    }
}

// master[slot] = sum of the partials of that slot: counts [rows][nb] followed by offset sums [nb]
struct MasterSlot {
    unsigned long long* cnt;
    unsigned long long* ds;
    int rows, n_parts;
    const unsigned long long* const* parts;
};
struct MasterSum {
    MasterSlot slot[3];
    int nb;
    int32_t* max_bin;
};

__global__ void master_sum_kernel(MasterSum M) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) *M.max_bin = 0;  // the finalisation raises it
    const MasterSlot S = M.slot[blockIdx.y];
    const long long nc = static_cast<long long>(S.rows) * M.nb;
    const long long n = nc + M.nb;
    for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        unsigned long long v = 0;
        for (int p = 0; p < S.n_parts; ++p) v += S.parts[p][e];
        if (e < nc) S.cnt[e] = v;
        else S.ds[e - nc] = v;
    }
}

void compose(Pose& P, const double* R, const double* t) {
    Pose o = P;
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c)
            P.R[3 * r + c] = R[3 * r] * o.R[c] + R[3 * r + 1] * o.R[3 + c] + R[3 * r + 2] * o.R[6 + c];
        P.t[r] = R[3 * r] * o.t[0] + R[3 * r + 1] * o.t[1] + R[3 * r + 2] * o.t[2] + t[r];
    }
}

}  // namespace

// tiles of a serving pair launch's CTA: a CTA lives for a few hundred microseconds at most
constexpr int kServeTilesPerCta = 2;

struct Assembly {
    Ctx C;  // C.stream: the stream of the request being enqueued (one of `streams`)
    cudaStream_t streams[2] = {nullptr, nullptr};  // [0] high priority, [1] low priority
    cudaEvent_t last = nullptr;                    // end of the last enqueued request
    bool has_last = false;
    std::vector<long long> move_pairs;             // pair evaluations of a move of each body
    ausaxs_hist_config cfg{};
    Structure S;  // the whole assembly: current coordinates; its plan's accumulators are the master
    int B = 0, N = 0, W = 0;
    std::vector<int> a_off, w_off;
    std::vector<std::array<double, 3>> c0;  // body centroids of the original coordinates
    std::vector<Pose> pose;
    DevBuf orig, part, tables, io;
    struct Part {
        int kind, k, l;  // kind 0: aa (k <= l), 1: aw (atoms of k x waters of l), 2: ww (k <= l)
        size_t off;      // byte offset in `part`
        int rows;
    };
    std::vector<Part> parts;
    struct Work {  // one pair launch over a set of partials
        size_t zero_off = 0;
        int n_zero = 0;
        PairLaunch L{};
        int grid = 0;
    };
    std::vector<Work> work;  // [B]: moves of body k; [B]: every partial (initial state)
    MasterSum msum{};
    int tile = 256;
    size_t smem = 0;
    int nq = 0;
    ausaxs_debye_params params{};
    bool fit = false;
    double *q_dev = nullptr, *I_dev = nullptr, *target_dev = nullptr, *err_dev = nullptr, *lsq_dev = nullptr;
    std::vector<double*> free_slots;  // pinned output slots [nq + 5]
    std::vector<double*> all_slots;
    size_t footprint = 0;

    ~Assembly() {
        cudaSetDevice(C.device);
        sync();
        for (double* p : all_slots) cudaFreeHost(p);
        if (C.h_stats) cudaFreeHost(C.h_stats);
        C.h_stats = nullptr;
        for (auto& st : streams)
            if (st) cudaStreamDestroy(st);
        if (last) cudaEventDestroy(last);
        C.stream = nullptr;
    }

    void sync() {
        for (auto& st : streams)
            if (st) cudaStreamSynchronize(st);
        if (has_last) cudaEventSynchronize(last);  // a request on the server's arrival-order stream
    }

    // the stream of a request with this priority, ordered after the assembly's previous request
    void select_stream(bool high) { select(streams[high ? 0 : 1]); }
    void select(cudaStream_t st) {
        if (has_last && st != C.stream) AUSAXS_CUDA(cudaStreamWaitEvent(st, last, 0));
        C.stream = st;
    }

    size_t block_bytes(int rows) const { return align_up((size_t)(rows + 1) * S.plan.nb * 8, 256); }

    void create(int device, int sms, const ausaxs_hist_config& c, int n_bodies, const float* atoms, const int64_t* aoff,
                const float* waters, const int64_t* woff, double margin, const double* q, int n_q,
                const ausaxs_debye_params& p, const double* target, const double* err, int slots) {
        if (c.manager != AUSAXS_MANAGER_FFAVG) throw Error{AUSAXS_ERR_ARGUMENT, "assemblies use the FFAVG manager"};
        if (n_bodies <= 0 || !aoff || !woff || !q || n_q <= 0 || slots <= 0 || !(margin >= 0))
            throw Error{AUSAXS_ERR_ARGUMENT, "bad assembly arguments"};
        C.device = device;
        C.sm_count = sms;
        int least = 0, greatest = 0;
        AUSAXS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        AUSAXS_CUDA(cudaStreamCreateWithPriority(&streams[0], cudaStreamNonBlocking, greatest));
        AUSAXS_CUDA(cudaStreamCreateWithPriority(&streams[1], cudaStreamNonBlocking, least));
        AUSAXS_CUDA(cudaEventCreateWithFlags(&last, cudaEventDisableTiming));
        C.stream = streams[1];
        C.own_stream = false;  // the streams belong to the assembly
        AUSAXS_CUDA(cudaMallocHost(&C.h_stats, sizeof(PrepStats)));
        cfg = c;
        B = n_bodies;
        for (int k = 0; k <= B; ++k) {
            a_off.push_back((int)aoff[k]);
            w_off.push_back((int)woff[k]);
            if (k && (aoff[k] < aoff[k - 1] || woff[k] < woff[k - 1])) throw Error{AUSAXS_ERR_ARGUMENT, "bad offsets"};
        }
        if (aoff[0] != 0 || woff[0] != 0 || aoff[B] > INT32_MAX || woff[B] > INT32_MAX)
            throw Error{AUSAXS_ERR_ARGUMENT, "bad offsets"};
        N = a_off[B];
        W = w_off[B];
        // body centroids (host), identity poses
        for (int k = 0; k < B; ++k) {
            std::array<double, 3> m{0, 0, 0};
            const int n = a_off[k + 1] - a_off[k];
            for (int i = a_off[k]; i < a_off[k + 1]; ++i)
                for (int d = 0; d < 3; ++d) m[d] += atoms[4 * (size_t)i + d];
            for (int d = 0; d < 3; ++d) m[d] = n ? m[d] / n : 0.0;
            c0.push_back(m);
            Pose id{};
            id.R[0] = id.R[4] = id.R[8] = 1.0;
            pose.push_back(id);
        }
        S.ctx = &C;
        S.load(atoms, N, waters, W, nullptr, 0, 1, true);
        S.dmax_extra = (float)margin;
        Plan& P = S.plan_for(cfg);
        const int nb = P.nb, T = S.T;
        // original coordinates (dense atom types), the source of every transform
        const size_t a_bytes = (size_t)std::max(1, N) * 16, w_bytes = (size_t)std::max(1, W) * 16;
        orig.ensure(align_up(a_bytes, 256) + w_bytes);
        AUSAXS_CUDA(cudaMemcpyAsync(orig.p, S.atoms_for_pairs(), (size_t)N * 16, cudaMemcpyDeviceToDevice, C.stream));
        if (W) AUSAXS_CUDA(cudaMemcpyAsync(orig.as<char>(align_up(a_bytes, 256)), S.raw_w.p, (size_t)W * 16,
                                           cudaMemcpyDeviceToDevice, C.stream));
        // partial blocks
        size_t off = 0;
        auto add = [&](int kind, int k, int l, int rows) {
            parts.push_back({kind, k, l, off, rows});
            off += block_bytes(rows);
        };
        for (int k = 0; k < B; ++k)
            for (int l = k; l < B; ++l) add(0, k, l, T * T);
        for (int k = 0; k < B; ++k)
            for (int l = 0; l < B; ++l) add(1, k, l, T);
        for (int k = 0; k < B; ++k)
            for (int l = k; l < B; ++l) add(2, k, l, 1);
        part.ensure(off + 256);
        const size_t counter_off = off;  // tile counter word after the blocks

        // pair jobs of every partial
        const float4* A = S.atoms_for_pairs();
        const float4* Wp = S.raw_w.as<float4>();
        auto spec_of = [&](const Part& pt) {
            JobSpec j{};
            unsigned long long* blk = part.as<unsigned long long>(pt.off);
            j.counts = blk;
            j.dsum = cfg.weighted_bins ? blk + (size_t)pt.rows * nb : nullptr;
            j.wsum = nullptr;
            j.rows = pt.rows;
            const int k = pt.k, l = pt.l;
            if (pt.kind == 0) {  // aa: body k atoms outer, body l atoms inner, rows of the full self loop
                j.A = A + a_off[k];
                j.na = a_off[k + 1] - a_off[k];
                j.B = A + a_off[l];
                j.nbp = a_off[l + 1] - a_off[l];
                j.self = k == l;
                j.rmode = kRowPair;
                j.a_base = a_off[k];
                j.b_base = a_off[l];
                j.tail_end = N;
                j.tail_from_outer = 1;
            } else if (pt.kind == 1) {  // aw: atoms of k outer, waters of l inner, rows over all waters
                j.A = A + a_off[k];
                j.na = a_off[k + 1] - a_off[k];
                j.B = Wp + w_off[l];
                j.nbp = w_off[l + 1] - w_off[l];
                j.self = 0;
                j.rmode = kRowOuter;
                j.a_base = a_off[k];
                j.b_base = w_off[l];
                j.tail_end = W;
                j.tail_from_outer = 0;
            } else {  // ww
                j.A = Wp + w_off[k];
                j.na = w_off[k + 1] - w_off[k];
                j.B = Wp + w_off[l];
                j.nbp = w_off[l + 1] - w_off[l];
                j.self = k == l;
                j.rmode = kRowSingle;
                j.a_base = w_off[k];
                j.b_base = w_off[l];
                j.tail_end = W;
                j.tail_from_outer = 1;
            }
            return j;
        };
        tile = P.tile;
        std::vector<PairJob> all_jobs;
        std::vector<ZeroRange> all_zero;
        work.resize(B + 1);
        int max_rows = 1;
        for (int k = 0; k <= B; ++k) {  // k == B: every partial
            Plan tmp;  // job-building view of the plan
            tmp.T = T;
            tmp.nb = nb;
            tmp.inv_w = P.inv_w;
            tmp.c = P.c;
            tmp.scale = P.scale;
            tmp.max_group_rows = P.max_group_rows;
            std::vector<ZeroRange> zr;
            for (const Part& pt : parts) {
                // every partial with the moved body, its self partials included: the moved coordinates are
                // rounded to float, so a few of its own pairs can change bins (the reference keeps them,
                // PartialHistogramManagerMT.cpp:118-125; recomputing keeps the master equal to a full
                // calculate_all() of the moved coordinates)
                const bool moved = k == B || pt.k == k || pt.l == k;
                if (!moved) continue;
                JobSpec j = spec_of(pt);
                if (j.na > 0 && j.nbp > 0 && !(j.self && j.na < 2)) tmp.specs.push_back(j);
                zr.push_back({part.as<unsigned long long>(pt.off), (long long)((pt.rows + 1) * (size_t)nb)});
            }
            zr.push_back({part.as<unsigned long long>(counter_off), 1});
            std::vector<PairJob> js[3];
            long long tiles[3] = {0, 0, 0};
            int rows[3] = {1, 1, 1};
            append_pair_jobs(tmp, tile, false, js, tiles, rows);
            Work& Wk = work[k];
            Wk.zero_off = all_zero.size();
            Wk.n_zero = (int)zr.size();
            all_zero.insert(all_zero.end(), zr.begin(), zr.end());
            Wk.L.n_jobs = (int)js[0].size();
            Wk.L.total_tiles = tiles[0];
            Wk.L.smem_rows = rows[0];
            Wk.L.smem_bins = nb;
            Wk.L.tile_counter = part.as<unsigned long long>(counter_off);
            Wk.L.overflow = P.dev.as<unsigned long long>(P.off_overflow);
            Wk.L.weighted = 0;
            Wk.L.wscale = nullptr;
            Wk.L.inv_w = P.inv_w;
            Wk.L.jobs = reinterpret_cast<const PairJob*>(all_jobs.size());  // index, rebased below
            all_jobs.insert(all_jobs.end(), js[0].begin(), js[0].end());
            max_rows = std::max(max_rows, rows[0]);
        }
        smem = pairhist_launch_smem(max_rows, nb, false, tile);
        // two thread groups per CTA (pairhist_groups): a tile of a move's short-lived CTAs takes half
        // the time, which shortens the last wave of a move (measured: the largest body's lone move
        // 1.43 -> 1.38 ms p50, 2.54 -> 2.21 ms max; saturated moves/s +3 %)
        for (Work& Wk : work) {
            Wk.L.dreg = pairhist_dreg(max_rows, nb, false, tile) ? 1 : 0;
            Wk.L.groups = Wk.L.dreg ? 1 : 2;
        }
        const int per_sm = pairhist_ctas_per_sm(smem, tile, pairhist_dreg(max_rows, nb, false, tile), false);
        // device tables: jobs, zero ranges, partial pointers of the master sum
        std::vector<const unsigned long long*> ptrs[3];
        for (const Part& pt : parts) ptrs[pt.kind].push_back(part.as<unsigned long long>(pt.off));
        const size_t jobs_bytes = align_up(sizeof(PairJob) * std::max<size_t>(1, all_jobs.size()), 256);
        const size_t zero_bytes = align_up(sizeof(ZeroRange) * all_zero.size(), 256);
        size_t ptr_off[3], toff = jobs_bytes + zero_bytes;
        for (int s = 0; s < 3; ++s) {
            ptr_off[s] = toff;
            toff += align_up(sizeof(void*) * std::max<size_t>(1, ptrs[s].size()), 256);
        }
        tables.ensure(toff);
        AUSAXS_CUDA(cudaMemcpy(tables.p, all_jobs.data(), sizeof(PairJob) * all_jobs.size(), cudaMemcpyHostToDevice));
        AUSAXS_CUDA(cudaMemcpy(tables.as<char>(jobs_bytes), all_zero.data(), sizeof(ZeroRange) * all_zero.size(),
                               cudaMemcpyHostToDevice));
        for (int s = 0; s < 3; ++s)
            AUSAXS_CUDA(cudaMemcpy(tables.as<char>(ptr_off[s]), ptrs[s].data(), sizeof(void*) * ptrs[s].size(),
                                   cudaMemcpyHostToDevice));
        for (Work& Wk : work) {
            Wk.L.jobs = tables.as<PairJob>() + reinterpret_cast<size_t>(Wk.L.jobs);
            Wk.zero_off = jobs_bytes + Wk.zero_off * sizeof(ZeroRange);
            // short-lived CTAs of kServeTilesPerCta tiles each (one tile per grab), at least one wave
            Wk.L.chunk = 1;
            Wk.L.max_grabs = kServeTilesPerCta;
            const long long need = (Wk.L.total_tiles + kServeTilesPerCta - 1) / kServeTilesPerCta;
            Wk.grid = (int)std::max<long long>(1, std::min<long long>(need, (long long)INT32_MAX));
            (void)per_sm;
        }
        // pair evaluations of a move of each body (the body against the rest, and its own pairs)
        const long long NW = (long long)N + W;
        for (int k = 0; k < B; ++k) {
            const long long nk = (long long)(a_off[k + 1] - a_off[k]) + (w_off[k + 1] - w_off[k]);
            move_pairs.push_back(nk * (NW - nk) + nk * (nk - 1) / 2);
        }
        const FinalizeFF& F = P.fin_ff;
        msum.nb = nb;
        msum.max_bin = F.max_bin;
        const unsigned long long* cnts[3] = {F.cnt_aa, F.cnt_aw, F.cnt_ww};
        const unsigned long long* dss[3] = {F.ds_aa, F.ds_aw, F.ds_ww};
        const int srows[3] = {T * T, T, 1};
        for (int s = 0; s < 3; ++s) {
            msum.slot[s].cnt = const_cast<unsigned long long*>(cnts[s]);
            msum.slot[s].ds = const_cast<unsigned long long*>(dss[s]);
            msum.slot[s].rows = srows[s];
            msum.slot[s].n_parts = (int)ptrs[s].size();
            msum.slot[s].parts = tables.as<const unsigned long long*>(ptr_off[s]);
        }
        // transform inputs and outputs
        nq = n_q;
        params = p;
        fit = target != nullptr;
        const size_t qb = align_up((size_t)nq * 8, 256);
        io.ensure(4 * qb + 256);
        q_dev = io.as<double>();
        I_dev = io.as<double>(qb);
        target_dev = io.as<double>(2 * qb);
        err_dev = io.as<double>(3 * qb);
        lsq_dev = io.as<double>(4 * qb);
        AUSAXS_CUDA(cudaMemcpy(q_dev, q, (size_t)nq * 8, cudaMemcpyHostToDevice));
        if (fit) {
            std::vector<double> e(nq, 1.0);
            if (err) std::copy(err, err + nq, e.begin());
            AUSAXS_CUDA(cudaMemcpy(target_dev, target, (size_t)nq * 8, cudaMemcpyHostToDevice));
            AUSAXS_CUDA(cudaMemcpy(err_dev, e.data(), (size_t)nq * 8, cudaMemcpyHostToDevice));
        }
        for (int k = 0; k < slots; ++k) {
            double* h = nullptr;
            AUSAXS_CUDA(cudaMallocHost(&h, sizeof(double) * (nq + 5)));
            all_slots.push_back(h);
            free_slots.push_back(h);
        }
        // every partial once (the initial state)
        AUSAXS_CUDA(cudaMemsetAsync(P.dev.as<char>(P.off_overflow), 0, 8, C.stream));
        enqueue_pairs(work[B]);
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
        footprint = S.raw_a.n + S.raw_w.n + S.raw_x.n + S.dense_a.n + S.meta.n + P.dev.n + orig.n + part.n + tables.n +
                    io.n + C.stats.n;
    }

    void enqueue_pairs(const Work& Wk) {
        zero_ranges_launch(tables.as<ZeroRange>(Wk.zero_off), Wk.n_zero, C.stream);
        C.check_launch("zero");
        if (Wk.L.n_jobs > 0) {
            pairhist_launch(Wk.L, tile, Wk.grid, smem, C.stream);
            C.check_launch("pairhist");
        }
    }

    // move body (or none: body < 0), then the master, I(q) and the fit into `slot` (async)
    void enqueue_request(int body, const double* R, const double* t, double* slot) {
        cudaStream_t s = C.stream;
        if (body >= 0) {
            compose(pose[body], R, t);
            const int na = a_off[body + 1] - a_off[body], nw = w_off[body + 1] - w_off[body];
            const size_t a_bytes = align_up((size_t)std::max(1, N) * 16, 256);
            if (na)
                transform_kernel<<<std::min(1024, (na + 255) / 256), 256, 0, s>>>(
                    orig.as<float4>() + a_off[body], const_cast<float4*>(S.atoms_for_pairs()) + a_off[body], na, pose[body]);
            if (nw)
                transform_kernel<<<std::min(1024, (nw + 255) / 256), 256, 0, s>>>(
                    orig.as<float4>(a_bytes) + w_off[body], S.raw_w.as<float4>() + w_off[body], nw, pose[body]);
            C.check_launch("transform");
            enqueue_pairs(work[body]);
        }
        const int blocks = (int)std::min<long long>(1024, ((long long)(S.T * S.T + 1) * S.plan.nb + 255) / 256);
        master_sum_kernel<<<dim3(blocks, 3), 256, 0, s>>>(msum);
        C.check_launch("master");
        ff_finalize_launch(S.plan.fin_ff, s);
        C.check_launch("finalize");
        DebyeArgs A = S.debye_args(cfg, q_dev, nq, params, I_dev, nullptr);
        A.fp64_columns = nullptr;
        // FP64 (precision 1), or the exact tensor-core contraction (3; 2 when it pays off) over tables
        // kept with the assembly's plan (made when its first request runs)
        run_debye(C, A, 1, S.plan.tc, params.precision, &S.plan.x, cfg.bin_width);
        if (fit) {
            lsq_launch(target_dev, I_dev, err_dev, nq, lsq_dev, s);
            C.check_launch("lsq");
        } else {
            AUSAXS_CUDA(cudaMemsetAsync(lsq_dev, 0, 5 * 8, s));
        }
        AUSAXS_CUDA(cudaMemcpyAsync(slot, I_dev, (size_t)nq * 8, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaMemcpyAsync(slot + nq, lsq_dev, 5 * 8, cudaMemcpyDeviceToHost, s));
    }
};

struct Server {
    int device = 0, sms = 148;
    long long budget = 0, used = 0;
    int max_inflight = 64, slots_per_assembly = 4;
    std::map<int, std::unique_ptr<Assembly>> asms;
    int next_id = 1;
    struct Req {
        int asm_id;
        cudaEvent_t ev;
        double* slot;
    };
    std::map<long long, Req> inflight;
    long long next_ticket = 1;
    std::vector<cudaEvent_t> events;
    long long high_priority_pairs = 0;  // moves of at most this many pairs run on high-priority streams
    // 0: every assembly's requests on its own two streams (concurrent; small moves at high priority);
    // k > 0: requests in submission order, round robin over k server streams (at most k moves share
    // the GPU; k = 1: each move has it alone).  Two lanes by default: a move waits for at most one
    // other, and the pair launches of two moves still fill each other's last waves.
    int policy = 2;
    std::vector<cudaStream_t> lanes;
    size_t next_lane = 0;

    // the median move size over the bodies of every admitted assembly
    void update_priority_threshold() {
        std::vector<long long> all;
        for (auto& a : asms) all.insert(all.end(), a.second->move_pairs.begin(), a.second->move_pairs.end());
        if (all.empty()) {
            high_priority_pairs = 0;
            return;
        }
        std::nth_element(all.begin(), all.begin() + all.size() / 2, all.end());
        high_priority_pairs = all[all.size() / 2];
    }

    ~Server() {
        cudaSetDevice(device);
        for (auto& r : inflight) cudaEventSynchronize(r.second.ev);
        for (auto& r : inflight) cudaEventDestroy(r.second.ev);
        for (auto e : events) cudaEventDestroy(e);
        asms.clear();
        for (auto st : lanes) cudaStreamDestroy(st);
    }

    Assembly& get(int id) {
        auto it = asms.find(id);
        if (it == asms.end()) throw Error{AUSAXS_ERR_NOT_FOUND, "no such assembly"};
        return *it->second;
    }

    // completes `ticket` if its event has fired: copies the outputs and frees the slot
    bool try_complete(long long ticket, double* Iq, double* fit5) {
        auto it = inflight.find(ticket);
        if (it == inflight.end()) throw Error{AUSAXS_ERR_NOT_FOUND, "no such request"};
        cudaError_t e = cudaEventQuery(it->second.ev);
        if (e == cudaErrorNotReady) return false;
        if (e != cudaSuccess) throw Error{AUSAXS_ERR_CUDA, std::string("request: ") + cudaGetErrorString(e)};
        Assembly& A = get(it->second.asm_id);
        if (Iq) std::copy(it->second.slot, it->second.slot + A.nq, Iq);
        if (fit5) std::copy(it->second.slot + A.nq, it->second.slot + A.nq + 5, fit5);
        A.free_slots.push_back(it->second.slot);
        events.push_back(it->second.ev);
        inflight.erase(it);
        return true;
    }
};

}  // namespace ausaxs_b200

using namespace ausaxs_b200;

struct ausaxs_gpu_server {
    Server impl;
};

extern "C" {

int ausaxs_gpu_server_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_inflight,
                             int32_t slots_per_assembly, ausaxs_gpu_server** out) {
    return guarded([&] {
        if (!out || hbm_budget_bytes <= 0 || max_inflight <= 0 || slots_per_assembly <= 0)
            throw Error{AUSAXS_ERR_ARGUMENT, "bad server arguments"};
        *out = nullptr;
        int n = 0;
        AUSAXS_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Error{AUSAXS_ERR_ARGUMENT, "no such CUDA device"};
        AUSAXS_CUDA(cudaSetDevice(device));
        auto* s = new ausaxs_gpu_server();
        s->impl.device = device;
        cudaDeviceGetAttribute(&s->impl.sms, cudaDevAttrMultiProcessorCount, device);
        s->impl.budget = hbm_budget_bytes;
        s->impl.max_inflight = max_inflight;
        s->impl.slots_per_assembly = slots_per_assembly;
        *out = s;
    });
}

int ausaxs_gpu_server_set_policy(ausaxs_gpu_server* s, int32_t policy) {
    return guarded([&] {
        if (!s || policy < 0 || policy > 16) throw Error{AUSAXS_ERR_ARGUMENT, "bad scheduling policy"};
        s->impl.policy = policy;
    });
}

int ausaxs_gpu_server_destroy(ausaxs_gpu_server* s) {
    return guarded([&] { delete s; });
}

int ausaxs_gpu_server_admit(ausaxs_gpu_server* s, const ausaxs_hist_config* cfg, int32_t n_bodies, const float* atoms,
                            const int64_t* atom_offsets, const float* waters, const int64_t* water_offsets,
                            double margin, const double* q, int32_t n_q, const ausaxs_debye_params* params,
                            const double* target, const double* target_err, int32_t* id, int64_t* footprint) {
    return guarded([&] {
        if (!s || !cfg || !id || !params) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        auto A = std::make_unique<Assembly>();
        A->create(S.device, S.sms, *cfg, n_bodies, atoms, atom_offsets, waters, water_offsets, margin, q, n_q, *params,
                  target, target_err, S.slots_per_assembly);
        if (footprint) *footprint = (int64_t)A->footprint;
        if (S.used + (long long)A->footprint > S.budget)
            throw Error{AUSAXS_ERR_CAPACITY, "the assembly's device footprint exceeds the server's free budget"};
        S.used += (long long)A->footprint;
        *id = S.next_id++;
        S.asms[*id] = std::move(A);
        S.update_priority_threshold();
    });
}

int ausaxs_gpu_server_release(ausaxs_gpu_server* s, int32_t id) {
    return guarded([&] {
        if (!s) throw Error{AUSAXS_ERR_ARGUMENT, "null server"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        Assembly& A = S.get(id);
        for (auto& r : S.inflight)
            if (r.second.asm_id == id) throw Error{AUSAXS_ERR_CAPACITY, "the assembly has requests in flight"};
        S.used -= (long long)A.footprint;
        S.asms.erase(id);
        S.update_priority_threshold();
    });
}

int ausaxs_gpu_server_usage(ausaxs_gpu_server* s, int64_t* used, int64_t* budget, int32_t* inflight) {
    return guarded([&] {
        if (!s) throw Error{AUSAXS_ERR_ARGUMENT, "null server"};
        if (used) *used = s->impl.used;
        if (budget) *budget = s->impl.budget;
        if (inflight) *inflight = (int32_t)s->impl.inflight.size();
    });
}

int ausaxs_gpu_server_submit(ausaxs_gpu_server* s, int32_t id, int32_t body, const double* R, const double* t,
                             int64_t* ticket) {
    return guarded([&] {
        if (!s || !ticket) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        Assembly& A = S.get(id);
        if (body >= A.B || body < -1) throw Error{AUSAXS_ERR_ARGUMENT, "no such body"};
        if (body >= 0 && (!R || !t)) throw Error{AUSAXS_ERR_ARGUMENT, "a move needs R and t"};
        if ((int)S.inflight.size() >= S.max_inflight || A.free_slots.empty())
            throw Error{AUSAXS_ERR_CAPACITY, "no free request slot"};
        double* slot = A.free_slots.back();
        cudaEvent_t ev;
        if (!S.events.empty()) {
            ev = S.events.back();
            S.events.pop_back();
        } else {
            AUSAXS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        }
        try {
            if (S.policy > 0) {
                while ((int)S.lanes.size() < S.policy) {
                    cudaStream_t st;
                    AUSAXS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                    S.lanes.push_back(st);
                }
                A.select(S.lanes[S.next_lane++ % S.policy]);
            } else {
                A.select_stream(body >= 0 && A.move_pairs[body] <= S.high_priority_pairs);
            }
            A.enqueue_request(body, R, t, slot);
            AUSAXS_CUDA(cudaEventRecord(A.last, A.C.stream));
            A.has_last = true;
            AUSAXS_CUDA(cudaEventRecord(ev, A.C.stream));
        } catch (...) {
            S.events.push_back(ev);
            throw;
        }
        A.free_slots.pop_back();
        *ticket = S.next_ticket++;
        S.inflight[*ticket] = Server::Req{id, ev, slot};
    });
}

int ausaxs_gpu_server_poll(ausaxs_gpu_server* s, int64_t ticket, int32_t* done, double* Iq, double* fit5) {
    return guarded([&] {
        if (!s || !done) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        AUSAXS_CUDA(cudaSetDevice(s->impl.device));
        *done = s->impl.try_complete(ticket, Iq, fit5) ? 1 : 0;
    });
}

int ausaxs_gpu_server_wait(ausaxs_gpu_server* s, int64_t ticket, int32_t timeout_ms, double* Iq, double* fit5) {
    return guarded([&] {
        if (!s) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        AUSAXS_CUDA(cudaSetDevice(s->impl.device));
        const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(std::max(0, timeout_ms));
        while (!s->impl.try_complete(ticket, Iq, fit5)) {
            if (std::chrono::steady_clock::now() >= until) throw Error{AUSAXS_ERR_TIMEOUT, "request not finished in time"};
            std::this_thread::yield();
        }
    });
}

int ausaxs_gpu_server_launch_count(ausaxs_gpu_server* s, int64_t* launches) {
    return guarded([&] {
        if (!s || !launches) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        long long n = 0;
        for (auto& a : s->impl.asms) n += a.second->C.launches;
        *launches = n;
    });
}

int ausaxs_gpu_server_completed(ausaxs_gpu_server* s, int64_t* tickets, int32_t capacity, int32_t* n) {
    return guarded([&] {
        if (!s || !n || (capacity > 0 && !tickets)) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        int k = 0;
        for (auto& r : S.inflight) {
            if (k >= capacity) break;
            cudaError_t e = cudaEventQuery(r.second.ev);
            if (e == cudaSuccess) tickets[k++] = r.first;
            else if (e != cudaErrorNotReady) throw Error{AUSAXS_ERR_CUDA, std::string("request: ") + cudaGetErrorString(e)};
        }
        *n = k;
    });
}

int ausaxs_gpu_server_body_center(ausaxs_gpu_server* s, int32_t id, int32_t body, double* c) {
    return guarded([&] {
        if (!s || !c) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Assembly& A = s->impl.get(id);
        if (body < 0 || body >= A.B) throw Error{AUSAXS_ERR_ARGUMENT, "no such body"};
        const Pose& P = A.pose[body];
        const auto& m = A.c0[body];
        for (int r = 0; r < 3; ++r) c[r] = P.R[3 * r] * m[0] + P.R[3 * r + 1] * m[1] + P.R[3 * r + 2] * m[2] + P.t[r];
    });
}

int ausaxs_gpu_server_coordinates(ausaxs_gpu_server* s, int32_t id, float* atoms_xyzw, float* waters_xyzw) {
    return guarded([&] {
        if (!s) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        Assembly& A = S.get(id);
        A.sync();
        if (atoms_xyzw && A.N)
            AUSAXS_CUDA(cudaMemcpy(atoms_xyzw, A.S.atoms_for_pairs(), (size_t)A.N * 16, cudaMemcpyDeviceToHost));
        if (waters_xyzw && A.W) AUSAXS_CUDA(cudaMemcpy(waters_xyzw, A.S.raw_w.p, (size_t)A.W * 16, cudaMemcpyDeviceToHost));
    });
}

int ausaxs_gpu_server_histogram(ausaxs_gpu_server* s, int32_t id, ausaxs_hist_result* out) {
    return guarded([&] {
        if (!s || !out) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        Server& S = s->impl;
        AUSAXS_CUDA(cudaSetDevice(S.device));
        Assembly& A = S.get(id);
        A.sync();
        A.S.read_histogram(A.cfg, out);
    });
}

}  // extern "C"
