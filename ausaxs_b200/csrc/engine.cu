// Host-side engine of the Debye hot path: structure upload, plan construction and kernel enqueue.
//
// The reference runs a histogram manager's calculate_all() as thread-pool tasks over 800-row
// chunks (SimpleCalculator.h:117-141, GeneralSettings.cpp:50) and keeps all results in host
// memory.  Here a structure is uploaded once; a Plan lays out every accumulator and output of a
// (structure, configuration) pair in one device allocation and records the launch shapes, so a
// profile is a fixed sequence of kernels with no allocation and no host round trip.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.cuh"

namespace ausaxs_b200 {

void DevBuf::ensure(size_t bytes) {
    if (bytes <= n) return;
    if (!owned) throw Error{AUSAXS_ERR_CAPACITY, "device buffer view too small"};
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    if (bytes == 0) return;
    AUSAXS_CUDA(cudaMalloc(&p, bytes));
    n = bytes;
}

DevBuf::~DevBuf() {
    if (p && owned) cudaFree(p);
}

PrepStats* Ctx::stats_slots(size_t n) {
    if (n > n_stats_many) {
        if (h_stats_many) {
            cudaStreamSynchronize(stream);  // earlier read-backs may still target the old slots
            cudaFreeHost(h_stats_many);
        }
        h_stats_many = nullptr;
        n_stats_many = 0;
        AUSAXS_CUDA(cudaMallocHost(&h_stats_many, sizeof(PrepStats) * n));
        n_stats_many = n;
    }
    return h_stats_many;
}

void Ctx::check_launch(const char* what) {
    ++launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{AUSAXS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}


void Ctx::time_begin(int cls, cudaEvent_t* ev) {
    *ev = nullptr;
    if (!timing) return;
    AUSAXS_CUDA(cudaEventCreate(ev));
    AUSAXS_CUDA(cudaEventRecord(*ev, stream));
    (void)cls;
}

void Ctx::time_end(int cls, cudaEvent_t start) {
    if (!timing || !start) return;
    cudaEvent_t stop;
    AUSAXS_CUDA(cudaEventCreate(&stop));
    AUSAXS_CUDA(cudaEventRecord(stop, stream));
    timed[cls].pending.emplace_back(start, stop);
}

void Ctx::time_collect() {
    AUSAXS_CUDA(cudaStreamSynchronize(stream));
    for (auto& t : timed) {
        for (auto& e : t.pending) {
            float ms = 0;
            AUSAXS_CUDA(cudaEventElapsedTime(&ms, e.first, e.second));
            t.ms += ms;
            t.count += 1;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        t.pending.clear();
    }
}

void Structure::load_begin(const float* atoms, int n_atoms, const float* waters, int n_waters, const float* exv,
                           int n_exv, int ff_typed_, bool host, PrepStats* h_stats, PrepStats* d_stats, int exv_host) {
    if (n_atoms < 0 || n_waters < 0 || n_exv < 0) throw Error{AUSAXS_ERR_ARGUMENT, "negative point count"};
    if ((n_atoms && !atoms) || (n_waters && !waters) || (n_exv && !exv)) throw Error{AUSAXS_ERR_ARGUMENT, "null point array"};
    Ctx& C = *ctx;
    cudaStream_t s = C.stream;
    ff_typed = ff_typed_;
    // new points: the lattice form of the dummies (and a plan that bins them with it) is rebuilt
    lat.tried = false;
    lat.usable = false;
    if (plan.lattice_grid > 0) plan.manager = 0;
    n_a = n_atoms;
    n_w = n_waters;
    n_x = n_exv;
    raw_a.ensure(align_up(std::max(1, n_a) * 16, 256));
    raw_w.ensure(align_up(std::max(1, n_w) * 16, 256));
    raw_x.ensure(align_up(std::max(1, n_x) * 16, 256));
    cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (n_a) AUSAXS_CUDA(cudaMemcpyAsync(raw_a.p, atoms, (size_t)n_a * 16, kind, s));
    if (n_w) AUSAXS_CUDA(cudaMemcpyAsync(raw_w.p, waters, (size_t)n_w * 16, kind, s));
    const bool x_host = exv_host < 0 ? host : exv_host != 0;
    if (n_x) AUSAXS_CUDA(cudaMemcpyAsync(raw_x.p, exv, (size_t)n_x * 16, x_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));

    PrepStats init{};
    for (int k = 0; k < 3; ++k) init.lo[k] = 0xffffffffu, init.hi[k] = 0;
    *h_stats = init;  // pinned: the copy below reads it asynchronously, the census result overwrites it
    AUSAXS_CUDA(cudaMemcpyAsync(d_stats, h_stats, sizeof(PrepStats), cudaMemcpyHostToDevice, s));
    census_launch(raw_a.as<float4>(), n_a, ff_typed, d_stats, C.sm_count, s);
    census_launch(raw_w.as<float4>(), n_w, 0, d_stats, C.sm_count, s);
    census_launch(raw_x.as<float4>(), n_x, 0, d_stats, C.sm_count, s);
    radius_launch(raw_a.as<float4>(), n_a, raw_w.as<float4>(), n_w, raw_x.as<float4>(), n_x, d_stats, C.sm_count, s);
    C.check_launch("census");
    AUSAXS_CUDA(cudaMemcpyAsync(h_stats, d_stats, sizeof(PrepStats), cudaMemcpyDeviceToHost, s));
}

void Structure::load_end(const PrepStats& st) {
    Ctx& C = *ctx;
    cudaStream_t s = C.stream;
    if (st.bad & 1u)
        throw Error{AUSAXS_ERR_FORM_FACTOR,
                    "an atom has a form-factor type outside [1, 15) (UNKNOWN or excluded volume); form factor "
                    "information is required for the selected excluded volume model"};
    if (st.bad & 2u) throw Error{AUSAXS_ERR_ARGUMENT, "non-finite coordinate"};
    if (n_a + n_w + n_x > 0) {
        double d2 = 0;
        for (int k = 0; k < 3; ++k) {
            lo[k] = ordered_to_float(st.lo[k]);
            hi[k] = ordered_to_float(st.hi[k]);
            double e = (double)hi[k] - (double)lo[k];
            d2 += e * e;
        }
        // every pair distance is at most the box diagonal and at most twice the radius about the box
        // centre (tight for globules and shells, where the diagonal is sqrt(3) times the diameter)
        double r2;
        std::memcpy(&r2, &st.r2, sizeof r2);
        const double bound = std::min(std::sqrt(d2), 2.0 * std::sqrt(r2));
        dmax = (float)(bound * (1 + 1e-6) + 1e-3);
    } else {
        dmax = 0;
    }
    int T_new = 0;
    for (int f = 0; f < kNff; ++f) ff_to_type[f] = -1;
    if (ff_typed) {
        for (int f = 1; f < kNff; ++f)
            if (st.mask & (1u << f)) {
                type_ff[T_new] = f;
                type_count[T_new] = st.count[f];
                ff_to_type[f] = T_new;
                ++T_new;
            }
    }
    T = T_new;
    meta.ensure(256);
    for (int k = 0; k < kNff; ++k) hmeta[k] = k < T ? type_count[k] : 0, hmeta[kNff + k] = ff_to_type[k];
    // pageable source: the call returns once the bytes are staged, so hmeta may change afterwards
    AUSAXS_CUDA(cudaMemcpyAsync(meta.p, hmeta, sizeof(hmeta), cudaMemcpyHostToDevice, s));
    if (ff_typed) {
        dense_a.ensure(align_up(std::max(1, n_a) * 16, 256));
        to_dense_launch(raw_a.as<float4>(), dense_a.as<float4>(), n_a, meta.as<int32_t>(kNff * 4), C.sm_count, s);
        C.check_launch("to_dense");
    }
}

void Structure::load(const float* atoms, int n_atoms, const float* waters, int n_waters, const float* exv, int n_exv,
                     int ff_typed_, bool host, int exv_host) {
    Ctx& C = *ctx;
    C.stats.ensure(sizeof(PrepStats));
    load_begin(atoms, n_atoms, waters, n_waters, exv, n_exv, ff_typed_, host, C.h_stats, C.stats.as<PrepStats>(), exv_host);
    AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    load_end(*C.h_stats);
}

static long long tri(long long t) { return t * (t + 1) / 2; }

namespace {
// y: range, x: chunk of the range
__global__ void zero_ranges_kernel(const ZeroRange* ranges) {
    const ZeroRange r = ranges[blockIdx.y];
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < r.words; k += (long long)gridDim.x * blockDim.x)
        r.p[k] = r.src ? r.src[k] : 0ull;
}
}  // namespace

void zero_ranges_launch(const ZeroRange* ranges_dev, int n, cudaStream_t s) {
    if (n > 0) zero_ranges_kernel<<<dim3(16, n), 256, 0, s>>>(ranges_dev);
}

void append_pair_jobs(const Plan& P, int tile, bool by_class, std::vector<PairJob> (&jobs)[3], long long (&tiles)[3],
                      int (&rows)[3], int max_rows, bool skip_lattice) {
    auto nt = [tile](int n) { return (n + tile - 1) / tile; };
    const int group_rows = max_rows > 0 ? max_rows : P.max_group_rows;
    for (const JobSpec& j : P.specs) {
        if (skip_lattice && j.lattice) continue;
        const long long t = j.self ? tri(nt(j.na)) : (long long)nt(j.na) * nt(j.nbp);
        for (int r0 = 0; r0 < j.rows; r0 += group_rows) {
            const int r1 = std::min(j.rows, r0 + group_rows);
            const int g = !by_class ? 0 : ((r1 - r0) == 1 ? 0 : ((r1 - r0) <= P.T ? 1 : 2));
            PairJob pj{};
            pj.A = j.A;
            pj.B = j.B;
            pj.na = j.na;
            pj.nb = j.nbp;
            pj.self = j.self;
            pj.row_mode = j.rmode;
            pj.types = P.T;
            pj.row_lo = r0;
            pj.row_hi = r1;
            pj.nbins = P.nb;
            pj.tiles_i = nt(j.na);
            pj.tiles_j = nt(j.nbp);
            pj.tile_begin = tiles[g];
            pj.tile_count = t;
            pj.inv_w = P.inv_w;
            pj.c = P.c;
            pj.scale = P.scale;
            pj.counts = j.counts + (size_t)r0 * P.nb;
            pj.dsum = r0 == 0 ? j.dsum : nullptr;
            pj.wsum = r0 == 0 ? j.wsum : nullptr;
            pj.wscale = 0;  // read from device memory by weighted launches
            pj.mult = j.mult;
            pj.a_base = j.a_base;
            pj.b_base = j.b_base;
            pj.tail_end = j.tail_end >= 0 ? j.tail_end : j.nbp;
            pj.tail_from_outer = j.tail_from_outer >= 0 ? j.tail_from_outer : j.self;
            jobs[g].push_back(pj);
            tiles[g] += t;
            rows[g] = std::max(rows[g], r1 - r0);
        }
    }
}

bool Structure::lattice_ready() {
    if (lat.tried) return lat.usable;
    lat.tried = true;
    lat.usable = false;
    if (n_x < kLatticeMinPoints) return false;
    Ctx& C = *ctx;
    cudaStream_t s = C.stream;
    lat.scratch.ensure(256);
    int* st = lat.scratch.as<int>();
    lattice_scan_launch(raw_x.as<float4>(), n_x, st, C.sm_count, s);
    C.check_launch("lattice scan");
    int h[8] = {};
    AUSAXS_CUDA(cudaMemcpyAsync(h, st, 8 * sizeof(int), cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    if (h[6]) return false;  // not every coordinate is a (modest) integer or integer + 1/2
    for (int k = 0; k < 3; ++k)
        if (((h[7] >> (2 * k)) & 3) == 3) return false;  // integers and half-integers on one axis
    LatticeGrid G;
    for (int k = 0; k < 3; ++k) G.lo[k] = h[k];
    G.lx = h[3] - h[0] + 1;
    G.ly = h[4] - h[1] + 1;
    G.lz = h[5] - h[2] + 1;
    G.words = (G.lx + 31) / 32;
    if (G.words > kLatticeMaxWords || (long long)G.ly * G.lz > (1ll << 20)) return false;
    lat.s2_max = (long long)(G.lx - 1) * (G.lx - 1) + (long long)(G.ly - 1) * (G.ly - 1) + (long long)(G.lz - 1) * (G.lz - 1);
    if (lat.s2_max >= (1ll << 24)) return false;  // the reference's float evaluation is exact below 2^24
    const size_t n_lines_all = (size_t)G.ly * G.lz;
    DevBuf bits;
    bits.ensure(n_lines_all * G.words * 4);
    AUSAXS_CUDA(cudaMemsetAsync(bits.p, 0, n_lines_all * G.words * 4, s));
    lat.lines.ensure(n_lines_all * G.words * 4);
    lat.table.ensure(n_lines_all * 4);
    int* info = st + 8;
    AUSAXS_CUDA(cudaMemsetAsync(info, 0, 2 * sizeof(int), s));
    lattice_build_launch(raw_x.as<float4>(), n_x, G.lo, G.lx, G.ly, G.lz, G.words, bits.as<uint32_t>(),
                         lat.lines.as<uint32_t>(), lat.table.as<int32_t>(), info, C.sm_count, s);
    C.check_launch("lattice build");
    AUSAXS_CUDA(cudaMemcpyAsync(h, info, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));  // also keeps `bits` alive until the build is done
    if (h[1]) return false;  // two dummies in one cell (or outside the scanned box)
    G.n_lines = h[0];
    G.lines = lat.lines.as<uint32_t>();
    G.table = lat.table.as<int32_t>();
    lat.G = G;
    lat.usable = true;
    return true;
}

Plan& Structure::plan_for(const ausaxs_hist_config& cfg) {
    Plan& P = plan;
    if (cfg.bin_width <= 0 || cfg.bin_count <= 0) throw Error{AUSAXS_ERR_ARGUMENT, "bin_width and bin_count must be positive"};
    const bool ff = cfg.manager == AUSAXS_MANAGER_FFAVG || cfg.manager == AUSAXS_MANAGER_FFEXPLICIT ||
                    cfg.manager == AUSAXS_MANAGER_FFGRID;
    if (!ff && cfg.manager != AUSAXS_MANAGER_MT) throw Error{AUSAXS_ERR_ARGUMENT, "unknown manager"};
    if (ff != (ff_typed != 0))
        throw Error{AUSAXS_ERR_ARGUMENT, ff ? "form-factor managers need form-factor typed atoms"
                                            : "the weighted manager needs weighted atoms"};
    const int weighted = cfg.weighted_bins ? 1 : 0;
    const float inv_w = (float)(1.0 / cfg.bin_width);
    int nb = (int)std::ceil((double)(dmax + dmax_extra) * inv_w) + 2;
    nb = std::max(nb, 11);
    nb = std::min(nb, cfg.bin_count);
    if (P.manager == cfg.manager && P.weighted == weighted && P.bin_count == cfg.bin_count &&
        P.bin_width == cfg.bin_width && P.n_a == n_a && P.n_w == n_w && P.n_x == n_x && P.T == T && P.nb >= nb &&
        P.nb <= nb + 64 && (cfg.manager != AUSAXS_MANAGER_FFGRID || n_x < kLatticeMinPoints || lat.tried))
        return P;

    Ctx& C = *ctx;
    P.manager = cfg.manager;
    P.weighted = weighted;
    P.bin_count = cfg.bin_count;
    P.bin_width = cfg.bin_width;
    P.n_a = n_a;
    P.n_w = n_w;
    P.n_x = n_x;
    P.T = T;
    P.nb = nb;
    P.inv_w = inv_w;
    P.c = (float)(1.0 / (double)inv_w);
    // offsets r in [-c/2 (1 + 2^-10), c/2 (1 + 2^-10)] map into [0, 2^16)
    P.scale = (float)(32768.0 / (double)P.c * (1.0 - 1.0 / 256));
    const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
    const bool mt = cfg.manager == AUSAXS_MANAGER_MT;
    const int n_x_eff = grid ? n_x : 0;

    long long biggest = std::max<long long>({(long long)n_a, (long long)n_w, (long long)n_x_eff});
    P.tile = biggest >= 16384 ? 512 : 256;
    // Type-pair rows whose 512-point layout holds the CTA to one per SM (register-held offset sums)
    // and that still fit with 1024-point tiles run 1024 threads per CTA: the same shared memory
    // then serves 32 warps per SM instead of 16 (every launch of the plan uses the tile size).
    if (P.tile == 512 && !mt) {
        const int rows_aa = T * T;
        if (pairhist_dreg(rows_aa, nb, false, 512) && pairhist_dreg(rows_aa, nb, false, 1024) &&
            pairhist_launch_smem(rows_aa, nb, false, 1024) <= kPairSmemCap)
            P.tile = 1024;
    }
    const int tile = P.tile;
    auto nt = [tile](int n) { return (n + tile - 1) / tile; };

    // job list: {A, na, B, nb, self, row mode, rows, counts slot, dsum slot, wsum slot}
    struct J {
        const float4* A;
        int na;
        const float4* B;
        int nbp;
        int self, rmode, rows;
        int slot;  // accumulator slot (aa, aw, ww, ax, wx, xx)
    };
    std::vector<J> js;
    const float4* A = atoms_for_pairs();
    const float4* W = raw_w.as<float4>();
    const float4* X = raw_x.as<float4>();
    if (mt) {
        js.push_back({A, n_a, A, n_a, 1, kRowSingle, 1, 0});
        js.push_back({W, n_w, A, n_a, 0, kRowSingle, 1, 1});  // waters outer, atoms inner (SimpleCalculator.h:187-205)
        js.push_back({W, n_w, W, n_w, 1, kRowSingle, 1, 2});
    } else {
        js.push_back({A, n_a, A, n_a, 1, kRowPair, T * T, 0});
        js.push_back({A, n_a, W, n_w, 0, kRowOuter, T, 1});  // atoms outer, waters inner (HistogramManagerMTFFAvg.cpp:236-254)
        js.push_back({W, n_w, W, n_w, 1, kRowSingle, 1, 2});
        if (grid) {
            js.push_back({A, n_a, X, n_x, 0, kRowOuter, T, 3});  // HistogramManagerMTFFGrid.cpp:86-104
            js.push_back({W, n_w, X, n_x, 0, kRowSingle, 1, 4});  // :106-124
            js.push_back({X, n_x, X, n_x, 1, kRowSingle, 1, 5});  // :66-84
        }
    }
    const int slots = 6;
    int slot_rows[slots] = {0, 0, 0, 0, 0, 0};
    for (auto& j : js) slot_rows[j.slot] = std::max(slot_rows[j.slot], j.rows);

    // on-chip budget: split rows of a job into groups when its [rows][nb] counts do not fit
    const int max_group_rows = pairhist_max_rows(nb, weighted && mt, tile == 1024 ? 1024 : 512);
    if (pairhist_launch_smem(1, nb, weighted && mt, 512) > kPairSmemCap)
        throw Error{AUSAXS_ERR_CAPACITY, "too many distance bins for the on-chip histogram"};

    // layout
    size_t off = 0;
    P.off_jobs = off;
    std::vector<PairJob> jobs;
    off += align_up(sizeof(PairJob) * 64, 256);
    P.off_acc = off;
    size_t slot_cnt[slots], slot_ds[slots], slot_ws[slots];
    for (int k = 0; k < slots; ++k) {
        slot_cnt[k] = off;
        off += align_up((size_t)std::max(1, slot_rows[k]) * nb * 8, 256);
        slot_ds[k] = off;
        off += align_up((size_t)nb * 8, 256);
        slot_ws[k] = off;
        off += align_up((size_t)nb * 8, 256);
    }
    P.off_counter = off;
    off += 256;
    P.off_overflow = off;
    off += 256;
    P.off_maxbin = off;
    off += 256;
    P.off_wscale = off;
    off += 256;
    P.off_self = off;
    off += 256;
    P.off_fp64cols = off;
    off += 256;
    P.acc_bytes = off - P.off_acc;
    const int R = mt ? 3 : ff_rows(T);
    P.R = R;
    P.off_H = off;
    off += align_up((size_t)R * nb * 8, 256);
    P.off_tot = off;
    off += align_up((size_t)nb * 8, 256);
    P.off_d = off;
    off += align_up((size_t)nb * 8, 256);
    P.off_dax = off;
    off += align_up((size_t)nb * 8, 256);
    P.off_dxx = off;
    off += align_up((size_t)nb * 8, 256);
    P.off_rows = off;
    off += align_up(sizeof(RowDesc) * R, 256);
    P.off_expand_aa = 0;  // host-layout expansion buffers: allocated on the first read-back
    P.off_expand_aw = align_up((size_t)kNff * kNff * nb * 8, 256);
    P.dev.ensure(off);
    char* base = P.dev.as<char>();

    // the dummies' self pairs (slot 5) by the lattice kernel when the dummies sit on the integer
    // lattice and the reference's two rounding rules agree on every squared offset (lattice.cu)
    P.lattice_grid = 0;
    bool use_lattice = false;
    if (grid && n_x >= kLatticeMinPoints && lattice_ready()) {
        const size_t lsm = lattice_smem_bytes(lat.G.n_lines, lattice_kernel_words(lat.G.words), lat.G.ly, lat.G.lz, nb);
        if (lsm <= kPairSmemCap) {
            use_lattice = true;
            P.lattice_smem = lsm;
            const int per_sm = std::max(1, std::min(2048 / (lattice_kernel_words(lat.G.words) <= 4 ? 1024 : kLatticeThreads),
                                                    (int)(233472 / (lsm + 1024))));
            P.lattice_grid = C.sm_count * per_sm;
        }
    }
    // passes of this structure with their accumulators
    P.specs.clear();
    P.pairs = 0;
    for (auto& j : js) {
        if (j.na == 0 || j.nbp == 0) continue;
        long long pairs = j.self ? (long long)j.na * (j.na - 1) / 2 : (long long)j.na * j.nbp;
        if (pairs == 0) continue;
        P.pairs += pairs;
        JobSpec sp{};
        sp.A = j.A;
        sp.na = j.na;
        sp.B = j.B;
        sp.nbp = j.nbp;
        sp.self = j.self;
        sp.rmode = j.rmode;
        sp.rows = j.rows;
        sp.counts = reinterpret_cast<unsigned long long*>(base + slot_cnt[j.slot]);
        // offset sums only feed the weighted d-axis; weight sums are the Simple histogram's values
        sp.dsum = weighted ? reinterpret_cast<unsigned long long*>(base + slot_ds[j.slot]) : nullptr;
        sp.wsum = mt ? reinterpret_cast<long long*>(base + slot_ws[j.slot]) : nullptr;
        sp.lattice = use_lattice && j.slot == 5;
        P.specs.push_back(sp);
    }
    P.max_group_rows = max_group_rows;
    if (use_lattice) {
        LatticeLaunch& LL = P.lattice;
        LL.G = lat.G;
        LL.nbins = nb;
        LL.inv_w = P.inv_w;
        LL.c = P.c;
        LL.scale = P.scale;
        LL.counts = reinterpret_cast<unsigned long long*>(base + slot_cnt[5]);
        LL.dsum = weighted ? reinterpret_cast<unsigned long long*>(base + slot_ds[5]) : nullptr;
        LL.overflow = reinterpret_cast<unsigned long long*>(base + P.off_overflow);
        LL.counter = reinterpret_cast<unsigned long long*>(base + P.off_counter) + 8;  // cleared with the accumulators
        LL.n_items = lat.G.lz * (2 * lat.G.ly - 1) * kLatticeChunks;
        LL.pts = raw_x.as<float4>();
        LL.n_pts = n_x;
        LL.tail_fix = lattice_rules_agree(lat.s2_max, inv_w) ? 0 : 1;
    }

    // Jobs split into launch groups by the rows they keep on chip: one-row jobs (ww, xx, wx and all
    // Simple jobs) run with a small footprint and high occupancy, multi-row jobs (aa, aw, ax) get the
    // shared memory they need.  Large structures: one launch per row class (1, T, T*T rows) so each
    // gets the occupancy its footprint allows; small ones: everything in one launch (launch latency
    // dominates).  Tiles are numbered per group.
    pair_sqrt_prepare(P.inv_w, nb);  // once per width and process: the Newton-Raphson root where it bins exactly
    const bool split = P.pairs >= 2000000000LL;
    std::vector<PairJob> group_jobs[3];
    long long group_tiles[3] = {0, 0, 0};
    int group_rows[3] = {1, 1, 1};
    append_pair_jobs(P, tile, split, group_jobs, group_tiles, group_rows, 0, true);
    if (group_jobs[0].size() + group_jobs[1].size() + group_jobs[2].size() > 64)
        throw Error{AUSAXS_ERR_CAPACITY, "too many row groups"};
    const bool w_launch = mt;  // Simple histograms always carry weight sums (values)
    P.n_launch = 0;
    P.total_tiles = 0;
    size_t job_off = P.off_jobs;
    for (int g = 0; g < 3; ++g) {
        if (group_jobs[g].empty()) continue;
        Plan::Group& G = P.group[P.n_launch++];
        G.tile = tile;
        G.smem = pairhist_launch_smem(group_rows[g], nb, w_launch, tile);
        const bool dreg = pairhist_dreg(group_rows[g], nb, w_launch, tile);
        const int groups = pairhist_groups(G.smem, tile, dreg, w_launch, group_tiles[g], C.sm_count);
        const int per_sm = pairhist_ctas_per_sm(G.smem, tile, dreg, w_launch, groups);
        G.grid = (int)std::min<long long>((long long)C.sm_count * per_sm, std::max<long long>(1, group_tiles[g]));
        PairLaunch& L = G.launch;
        L.groups = groups;
        L.jobs = reinterpret_cast<const PairJob*>(base + job_off);
        L.n_jobs = (int)group_jobs[g].size();
        L.total_tiles = group_tiles[g];
        L.chunk = (int)std::max<long long>(1, std::min<long long>(8, group_tiles[g] / ((long long)G.grid * 8)));
        L.smem_rows = group_rows[g];
        L.smem_bins = nb;
        L.tile_counter = reinterpret_cast<unsigned long long*>(base + P.off_counter) + g;
        L.overflow = reinterpret_cast<unsigned long long*>(base + P.off_overflow);
        L.weighted = w_launch;
        L.dreg = pairhist_dreg(group_rows[g], nb, w_launch, tile) ? 1 : 0;
        L.wscale = reinterpret_cast<const float*>(base + P.off_wscale);
        L.inv_w = P.inv_w;
        AUSAXS_CUDA(cudaMemcpyAsync(base + job_off, group_jobs[g].data(), sizeof(PairJob) * group_jobs[g].size(),
                                    cudaMemcpyHostToDevice, C.stream));  // pageable: staged on return
        job_off += sizeof(PairJob) * group_jobs[g].size();
        P.total_tiles += group_tiles[g];
    }

    // finalisation
    auto cnt = [&](int k) { return reinterpret_cast<const unsigned long long*>(base + slot_cnt[k]); };
    auto ds = [&](int k) { return reinterpret_cast<const unsigned long long*>(base + slot_ds[k]); };
    if (mt) {
        FinalizeMT& F = P.fin_mt;
        F.nb = nb;
        F.c_aa = cnt(0);
        F.c_aw = cnt(1);
        F.c_ww = cnt(2);
        F.ds_aa = ds(0);
        F.ds_aw = ds(1);
        F.ds_ww = ds(2);
        F.w_aa = reinterpret_cast<const long long*>(base + slot_ws[0]);
        F.w_aw = reinterpret_cast<const long long*>(base + slot_ws[1]);
        F.w_ww = reinterpret_cast<const long long*>(base + slot_ws[2]);
        F.wscale = reinterpret_cast<const float*>(base + P.off_wscale);
        F.self_aa = reinterpret_cast<const double*>(base + P.off_self);
        F.self_ww = reinterpret_cast<const double*>(base + P.off_self) + 1;
        F.bin_width = cfg.bin_width;
        F.c = P.c;
        F.scale = P.scale;
        F.weighted = weighted;
        F.max_bin = reinterpret_cast<int32_t*>(base + P.off_maxbin);
        F.H = reinterpret_cast<double*>(base + P.off_H);
        F.tot = reinterpret_cast<double*>(base + P.off_tot);
        F.d_axis = reinterpret_cast<double*>(base + P.off_d);
    } else {
        FinalizeFF& F = P.fin_ff;
        F.kind = cfg.manager;
        F.T = T;
        F.nb = nb;
        F.n_a = n_a;
        F.n_w = n_w;
        F.n_x = n_x_eff;
        F.type_count = meta.as<int32_t>();
        F.ff_to_type = meta.as<int32_t>(kNff * 4);
        F.cnt_aa = cnt(0);
        F.cnt_aw = cnt(1);
        F.cnt_ww = cnt(2);
        F.cnt_ax = cnt(3);
        F.cnt_wx = cnt(4);
        F.cnt_xx = cnt(5);
        F.ds_aa = ds(0);
        F.ds_aw = ds(1);
        F.ds_ww = ds(2);
        F.ds_ax = ds(3);
        F.ds_wx = ds(4);
        F.ds_xx = ds(5);
        F.z_exv = cfg.z_exv;
        F.bin_width = cfg.bin_width;
        F.c = P.c;
        F.scale = P.scale;
        F.weighted = weighted;
        F.max_bin = reinterpret_cast<int32_t*>(base + P.off_maxbin);
        F.H = reinterpret_cast<double*>(base + P.off_H);
        F.tot = reinterpret_cast<double*>(base + P.off_tot);
        F.d_axis = reinterpret_cast<double*>(base + P.off_d);
        F.d_axis_ax = grid ? reinterpret_cast<double*>(base + P.off_dax) : nullptr;
        F.d_axis_xx = grid ? reinterpret_cast<double*>(base + P.off_dxx) : nullptr;
    }

    // row descriptors of the Debye transform
    std::vector<RowDesc> rd(R);
    if (mt) {
        rd[0] = {0, kRowSAA, 0, 0};
        rd[1] = {0, kRowSAW, 0, 0};
        rd[2] = {0, kRowSWW, 0, 0};
    } else {
        int g_ax = grid ? 1 : 0, g_xx = grid ? 2 : 0;
        // FFExplicit: the aa and aw rows also feed the exv profiles; the exv marginal rows are unused
        const bool ex = cfg.manager == AUSAXS_MANAGER_FFEXPLICIT;
        for (int a = 0; a < T; ++a)
            for (int b = 0; b < T; ++b) rd[a * T + b] = {0, ex ? kRowEAA : kRowAA, type_ff[a], type_ff[b]};
        for (int a = 0; a < T; ++a) rd[T * T + a] = {g_ax, ex ? kRowZero : kRowAX, type_ff[a], kExv};
        rd[T * T + T] = {g_xx, ex ? kRowZero : kRowXX, kExv, kExv};
        for (int a = 0; a < T; ++a) rd[T * T + T + 1 + a] = {0, ex ? kRowEAW : kRowAW, type_ff[a], kWater};
        rd[T * T + 2 * T + 1] = {g_ax, ex ? kRowZero : kRowWX, kExv, kWater};
        rd[T * T + 2 * T + 2] = {0, kRowWW, kWater, kWater};
    }
    AUSAXS_CUDA(cudaMemcpyAsync(base + P.off_rows, rd.data(), sizeof(RowDesc) * R, cudaMemcpyHostToDevice, C.stream));
    P.rows_host = rd;
    return P;
}

void Structure::enqueue_histogram(const ausaxs_hist_config& cfg) {
    Plan& P = plan_for(cfg);
    Ctx& C = *ctx;
    cudaStream_t s = C.stream;
    char* base = P.dev.as<char>();
    AUSAXS_CUDA(cudaMemsetAsync(base + P.off_acc, 0, P.acc_bytes, s));
    const bool mt = cfg.manager == AUSAXS_MANAGER_MT;
    if (mt) {
        weight_scale_launch(raw_a.as<float4>(), n_a, raw_w.as<float4>(), n_w, reinterpret_cast<float*>(base + P.off_wscale), s);
        weight_square_sum_launch(raw_a.as<float4>(), n_a, reinterpret_cast<double*>(base + P.off_self), s);
        weight_square_sum_launch(raw_w.as<float4>(), n_w, reinterpret_cast<double*>(base + P.off_self) + 1, s);
        C.check_launch("weights");
    }
    for (int g = 0; g < P.n_launch; ++g) {
        const Plan::Group& G = P.group[g];
        cudaEvent_t ev;
        C.time_begin(0, &ev);
        pairhist_launch(G.launch, G.tile, G.grid, G.smem, s);
        C.check_launch("pairhist");
        C.time_end(0, ev);
    }
    if (P.lattice_grid > 0) {
        cudaEvent_t ev;
        C.time_begin(6, &ev);
        lattice_launch(P.lattice, P.lattice_grid, P.lattice_smem, s);
        C.check_launch("lattice");
        C.time_end(6, ev);
    }
    cudaEvent_t evf;
    C.time_begin(1, &evf);
    if (mt) mt_finalize_launch(P.fin_mt, s);
    else ff_finalize_launch(P.fin_ff, s);
    C.check_launch("finalize");
    C.launches += 1;  // finalize is two kernels
    C.time_end(1, evf);
}

DebyeArgs Structure::debye_args(const ausaxs_hist_config& cfg, const double* q_dev, int nq, const ausaxs_debye_params& p,
                                double* Iq_dev, double* prof_dev) {
    Plan& P = plan;
    char* base = P.dev.as<char>();
    DebyeArgs A{};
    A.R = P.R;
    A.nb = P.nb;
    A.H = reinterpret_cast<const double*>(base + P.off_H);
    A.axis0 = reinterpret_cast<const double*>(base + P.off_d);
    const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
    A.axis1 = grid ? reinterpret_cast<const double*>(base + P.off_dax) : A.axis0;
    A.axis2 = grid ? reinterpret_cast<const double*>(base + P.off_dxx) : A.axis0;
    A.max_bin = reinterpret_cast<const int32_t*>(base + P.off_maxbin);
    A.rows = reinterpret_cast<const RowDesc*>(base + P.off_rows);
    A.overflow = reinterpret_cast<const unsigned long long*>(base + P.off_overflow);
    A.exv_model = grid ? 1 : (cfg.manager == AUSAXS_MANAGER_FFEXPLICIT ? 2 : 0);
    A.cw = p.cw;
    A.cx = p.cx;
    A.crho = p.crho;
    A.dw_atomic = p.dw_atomic;
    A.dw_exv = p.dw_exv;
    A.grid_volume = p.grid_width * p.grid_width * p.grid_width;
    A.q = q_dev;
    A.nq = nq;
    A.sinqd_tc = nullptr;
    A.bound_tc = nullptr;
    A.tolerance = p.tolerance > 0 ? p.tolerance : 1e-5;
    A.fp64_columns = reinterpret_cast<int32_t*>(base + P.off_fp64cols);
    A.Iq = Iq_dev;
    A.profiles = prof_dev;
    return A;
}

void Structure::enqueue_debye(const ausaxs_hist_config& cfg, const double* q_dev, int nq, const ausaxs_debye_params& p,
                              double* Iq_dev, double* prof_dev) {
    DebyeArgs A = debye_args(cfg, q_dev, nq, p, Iq_dev, prof_dev);
    run_debye(*ctx, A, cfg.manager == AUSAXS_MANAGER_FFGRID ? 7 : 1, plan.tc, p.precision, &plan.x, cfg.bin_width);
}

// The exact tensor-core transform of A's rows: buffers (re)made when the shape changes, the tables
// whenever the q values change (checked on the device); fills A's x fields.  false: not launched.
static bool enqueue_debye_x(Ctx& C, DebyeArgs& A, XBufs& X, double w) {
    cudaStream_t s = C.stream;
    XPlan& XP = X.plan;
    if (X.q != A.q || X.nq != A.nq || X.qmax < 0) {
        std::vector<double> hq(A.nq);
        AUSAXS_CUDA(cudaMemcpyAsync(hq.data(), A.q, sizeof(double) * A.nq, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaStreamSynchronize(s));
        double qmax = 0;
        for (double v : hq) qmax = std::max(qmax, std::fabs(v));
        X.qmax = qmax;
    }
    const int K = debye_x_order(X.qmax, w);
    const bool same = X.H == A.H && X.q == A.q && X.R == A.R && X.nb == A.nb && X.nq == A.nq && X.w == w && XP.K == K;
    if (!same) {
        XP.w = w;
        XP.nq = A.nq;
        XP.K = K;
        XP.nch = std::max(1, (A.nb + kXChunk - 1) / kXChunk);
        XP.n_rows = A.R;
        const int tiles = (A.R + 127) / 128;
        const long long qt = (A.nq + kXQTile - 1) / kXQTile;
        int splits = (XP.nch + debye_x_max_chunks(K) - 1) / debye_x_max_chunks(K);
        while (splits < XP.nch && qt * tiles * splits < 2LL * C.sm_count) ++splits;
        XP.cps = (XP.nch + splits - 1) / splits;
        XP.splits = (XP.nch + XP.cps - 1) / XP.cps;
        X.table.ensure(debye_x_table_bytes(A.nq, XP.nch, K));
        const size_t ncp = debye_x_cpart_doubles(A.nq, XP.nch);
        X.cpart.ensure(sizeof(double) * ncp);
        X.qcache.ensure(sizeof(double) * A.nq);
        AUSAXS_CUDA(cudaMemsetAsync(X.qcache.p, 0xff, sizeof(double) * A.nq, s));  // NaN: tables made on first use
        X.flags.ensure(256);
        AUSAXS_CUDA(cudaMemsetAsync(X.flags.p, 0, 256, s));
        const size_t nv = (size_t)XP.splits * A.R * A.nq, ne = (size_t)XP.splits * A.R;
        X.planes.ensure(sizeof(double) * (nv + 3 * ne));
        // rows: their distance axes from the row descriptors
        std::vector<RowDesc> rd(A.R);
        AUSAXS_CUDA(cudaMemcpyAsync(rd.data(), A.rows, sizeof(RowDesc) * A.R, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaStreamSynchronize(s));
        double* v = X.planes.as<double>();
        double* e1 = v + nv;
        double* e0 = e1 + ne;
        double* ha = e0 + ne;
        const double* axes[3] = {A.axis0, A.axis1 ? A.axis1 : A.axis0, A.axis2 ? A.axis2 : A.axis0};
        std::vector<XRow> rows(A.R);
        for (int r = 0; r < A.R; ++r) {
            XRow& xr = rows[r];
            xr = XRow{};
            xr.H = A.H + (size_t)r * A.nb;
            xr.axis = axes[std::min(2, std::max(0, rd[r].group))];
            xr.max_bin = A.max_bin;
            xr.out = v + (size_t)r * A.nq;
            xr.e1 = e1 + r;
            xr.e0 = e0 + r;
            xr.habs = ha + r;
            xr.out_z = (long long)A.R * A.nq;
            xr.e_z = A.R;
        }
        X.rows.ensure(sizeof(XRow) * A.R);
        AUSAXS_CUDA(cudaMemcpyAsync(X.rows.p, rows.data(), sizeof(XRow) * A.R, cudaMemcpyHostToDevice, s));
        std::vector<long long> toff(tiles);
        for (int t = 0; t < tiles; ++t) toff[t] = (long long)t * XP.nch * K * (long long)debye_x_block_bytes();
        X.adig.ensure((size_t)tiles * XP.nch * K * debye_x_block_bytes());
        X.tile_off.ensure(sizeof(long long) * tiles);
        AUSAXS_CUDA(cudaMemcpyAsync(X.tile_off.p, toff.data(), sizeof(long long) * tiles, cudaMemcpyHostToDevice, s));
        X.row_scale.ensure(sizeof(double) * A.R);
        AUSAXS_CUDA(cudaStreamSynchronize(s));  // the host staging vectors end here
        XP.rows = X.rows.as<XRow>();
        XP.table = X.table.as<unsigned char>();
        XP.cpart = X.cpart.as<double>();
        XP.q_cached = X.qcache.as<double>();
        XP.flags = X.flags.as<int32_t>();
        XP.adig = X.adig.as<unsigned char>();
        XP.tile_off = X.tile_off.as<long long>();
        XP.row_scale = X.row_scale.as<double>();
        X.H = A.H;
        X.q = A.q;
        X.R = A.R;
        X.nb = A.nb;
        X.nq = A.nq;
        X.w = w;
    }
    if (!debye_x_enqueue(XP, A.q, s)) return false;
    C.check_launch("debye_x");
    C.launches += 4;  // five kernels
    const size_t nv = (size_t)XP.splits * A.R * A.nq, ne = (size_t)XP.splits * A.R;
    double* v = X.planes.as<double>();
    A.x_v = v;
    A.x_e1 = v + nv;
    A.x_e0 = v + nv + ne;
    A.x_habs = v + nv + 2 * ne;
    A.x_splits = XP.splits;
    A.x_cpart = X.cpart.as<double>();
    A.x_nch = XP.nch;
    A.x_nqp = (int)(debye_x_cpart_doubles(A.nq, XP.nch) / XP.nch);
    A.x_K = XP.K;
    A.x_ctr = debye_x_trunc(XP.K, w);
    A.tc_error = X.flags.as<int32_t>() + 1;
    return true;
}

int run_debye(Ctx& C, DebyeArgs& A, int groups_present, DevBuf& tc, int precision, XBufs* xb, double w) {
    precision = debye_precision(precision, A.R, A.nb, A.nq);
    if (precision == 3 && (!xb || !(w > 0))) precision = 1;
    if (A.nq <= 0) return precision;
    cudaStream_t s = C.stream;
    if (precision == 3) {
        cudaEvent_t ev;
        C.time_begin(3, &ev);
        if (!enqueue_debye_x(C, A, *xb, w)) precision = 1;
        C.time_end(3, ev);
    }
    if (precision == 0) {
        // split-BF16 tensor-core contraction for every q, FP64 re-evaluation of the flagged ones
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, C.device);
        const int splits = debye_tc_splits(A.R, A.nb, A.nq, sms, __builtin_popcount((unsigned)groups_present));
        const size_t plane = (size_t)A.R * A.nq;
        const size_t n = (size_t)splits * plane;
        const size_t bytes_v = align_up(n * 4, 256), bytes_h = align_up((size_t)splits * A.R * 4, 256);
        tc.ensure(2 * bytes_v + bytes_h + 256);
        float* sq = tc.as<float>();
        float* bd = reinterpret_cast<float*>(tc.as<char>() + bytes_v);
        float* ha = reinterpret_cast<float*>(tc.as<char>() + 2 * bytes_v);
        int32_t* flag = reinterpret_cast<int32_t*>(tc.as<char>() + 2 * bytes_v + bytes_h);
        AUSAXS_CUDA(cudaMemsetAsync(flag, 0, 4, s));
        TcArgs T{};
        T.R = A.R;
        T.nb = A.nb;
        T.nq = A.nq;
        T.H = A.H;
        T.axis0 = A.axis0;
        T.axis1 = A.axis1;
        T.axis2 = A.axis2;
        T.rows = A.rows;
        T.max_bin = A.max_bin;
        T.q = A.q;
        T.groups_present = groups_present;
        T.splits = splits;
        T.sinqd = sq;
        T.bound = bd;
        T.habs = ha;
        T.error_flag = flag;
        cudaEvent_t ev;
        C.time_begin(3, &ev);
        const bool ok = debye_tc_launch(T, s);
        if (ok) C.check_launch("debye_tc");
        C.time_end(3, ev);
        if (ok) {
            A.sinqd_tc = sq;
            A.bound_tc = bd;
            A.habs_tc = ha;
            A.tc_splits = splits;
            A.tc_error = flag;
        }
    }
    cudaEvent_t ev;
    C.time_begin(2, &ev);
    debye_fp64_launch(A, s);
    C.check_launch("debye");
    C.time_end(2, ev);
    return precision;
}

void Structure::read_histogram(const ausaxs_hist_config& cfg, ausaxs_hist_result* out) {
    Plan& P = plan;
    Ctx& C = *ctx;
    cudaStream_t s = C.stream;
    char* base = P.dev.as<char>();
    struct {
        int32_t mb;
        int32_t pad;
        unsigned long long overflow;
    } hdr;
    AUSAXS_CUDA(cudaMemcpyAsync(&hdr.mb, base + P.off_maxbin, 4, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaMemcpyAsync(&hdr.overflow, base + P.off_overflow, 8, cudaMemcpyDeviceToHost, s));
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    const int mb = hdr.mb;
    const size_t nb = P.nb;
    out->max_bin = mb;
    out->pairs = P.pairs;
    out->overflow_pairs = (int64_t)hdr.overflow;
    const double* H = reinterpret_cast<const double*>(base + P.off_H);
    auto d2h = [&](double* dst, const void* src, size_t n) {
        if (dst && n) AUSAXS_CUDA(cudaMemcpyAsync(dst, src, n * 8, cudaMemcpyDeviceToHost, s));
    };
    if (cfg.manager == AUSAXS_MANAGER_MT) {
        d2h(out->aa, H, mb);
        d2h(out->aw, H + nb, mb);
        d2h(out->ww, H + 2 * nb, mb);
    } else {
        P.expand.ensure(P.off_expand_aw + align_up((size_t)kNff * nb * 8, 256));
        double* eaa = P.expand.as<double>(P.off_expand_aa);
        double* eaw = P.expand.as<double>(P.off_expand_aw);
        ff_expand_launch(P.fin_ff, eaa, eaw, mb, s);
        C.check_launch("expand");
        d2h(out->aa, eaa, (size_t)kNff * kNff * mb);
        d2h(out->aw, eaw, (size_t)kNff * mb);
        d2h(out->ww, H + (size_t)(ff_rows(P.T) - 1) * nb, mb);
        if (cfg.manager == AUSAXS_MANAGER_FFGRID) {
            d2h(out->d_axis_ax, base + P.off_dax, mb);
            d2h(out->d_axis_xx, base + P.off_dxx, mb);
        }
    }
    d2h(out->tot, base + P.off_tot, mb);
    d2h(out->d_axis, base + P.off_d, mb);
    AUSAXS_CUDA(cudaStreamSynchronize(s));
    if (hdr.overflow)
        throw Error{AUSAXS_ERR_BIN_OVERFLOW, "pair distances beyond bin_count * bin_width; increase settings::axes::bin_count"};
}

HostDebye upload_host_histogram(Ctx& C, const ausaxs_hist_config& cfg, const ausaxs_hist_result& h, const double* q,
                                int nq, const ausaxs_debye_params& p, size_t extra_bytes) {
    const int mb = h.max_bin;
    if (mb <= 0 || !h.d_axis || !h.aa || !h.aw || !h.ww) throw Error{AUSAXS_ERR_ARGUMENT, "incomplete histogram"};
    const bool mt = cfg.manager == AUSAXS_MANAGER_MT;
    const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
    if (grid && (!h.d_axis_ax || !h.d_axis_xx)) throw Error{AUSAXS_ERR_ARGUMENT, "grid histogram without ax/xx axes"};
    std::vector<double> H;
    std::vector<RowDesc> rd;
    auto row = [&](const double* src, RowDesc d) {
        H.insert(H.end(), src, src + mb);
        rd.push_back(d);
    };
    if (mt) {
        row(h.aa, {0, kRowSAA, 0, 0});
        row(h.aw, {0, kRowSAW, 0, 0});
        row(h.ww, {0, kRowSWW, 0, 0});
    } else {
        auto nonzero = [mb](const double* r) {
            for (int b = 0; b < mb; ++b)
                if (r[b] != 0) return true;
            return false;
        };
        std::vector<int> types;
        for (int f = 1; f < kNff; ++f) {
            bool used = nonzero(h.aw + (size_t)f * mb) || nonzero(h.aa + (size_t)(f * kNff) * mb);
            for (int g = 1; g < kNff && !used; ++g) used = nonzero(h.aa + (size_t)(f * kNff + g) * mb) || nonzero(h.aa + (size_t)(g * kNff + f) * mb);
            if (used) types.push_back(f);
        }
        int g_ax = grid ? 1 : 0, g_xx = grid ? 2 : 0;
        if (cfg.manager == AUSAXS_MANAGER_FFEXPLICIT) {
            for (int a : types)
                for (int b : types) row(h.aa + (size_t)(a * kNff + b) * mb, {0, kRowEAA, a, b});
            for (int a : types) row(h.aw + (size_t)a * mb, {0, kRowEAW, a, kWater});
        } else {
            for (int a : types)
                for (int b : types) row(h.aa + (size_t)(a * kNff + b) * mb, {0, kRowAA, a, b});
            for (int a : types) row(h.aa + (size_t)(a * kNff + kExv) * mb, {g_ax, kRowAX, a, kExv});
            row(h.aa, {g_xx, kRowXX, kExv, kExv});
            for (int a : types) row(h.aw + (size_t)a * mb, {0, kRowAW, a, kWater});
            row(h.aw, {g_ax, kRowWX, kExv, kWater});
        }
        row(h.ww, {0, kRowWW, kWater, kWater});
    }
    const int R = (int)rd.size();
    if (R > 264) throw Error{AUSAXS_ERR_CAPACITY, "too many histogram rows"};
    size_t off_H = 0, off_ax0 = align_up((size_t)R * mb * 8, 256);
    size_t off_ax1 = off_ax0 + align_up((size_t)mb * 8, 256), off_ax2 = off_ax1 + align_up((size_t)mb * 8, 256);
    size_t off_rows = off_ax2 + align_up((size_t)mb * 8, 256), off_mb = off_rows + align_up(sizeof(RowDesc) * R, 256);
    size_t off_q = off_mb + 256, off_I = off_q + align_up((size_t)nq * 8, 256), off_P = off_I + align_up((size_t)nq * 8, 256);
    size_t off_E = off_P + align_up((size_t)nq * 6 * 8, 256);
    size_t off_X = off_E + align_up((size_t)nq * 8, 256);
    size_t total = off_X + align_up(extra_bytes, 256);
    C.io.ensure(total);
    char* base = C.io.as<char>();
    cudaStream_t s = C.stream;
    AUSAXS_CUDA(cudaMemcpyAsync(base + off_H, H.data(), H.size() * 8, cudaMemcpyHostToDevice, s));
    AUSAXS_CUDA(cudaMemcpyAsync(base + off_ax0, h.d_axis, (size_t)mb * 8, cudaMemcpyHostToDevice, s));
    if (grid) {
        AUSAXS_CUDA(cudaMemcpyAsync(base + off_ax1, h.d_axis_ax, (size_t)mb * 8, cudaMemcpyHostToDevice, s));
        AUSAXS_CUDA(cudaMemcpyAsync(base + off_ax2, h.d_axis_xx, (size_t)mb * 8, cudaMemcpyHostToDevice, s));
    }
    AUSAXS_CUDA(cudaMemcpyAsync(base + off_rows, rd.data(), sizeof(RowDesc) * R, cudaMemcpyHostToDevice, s));
    int32_t mbv = mb;
    AUSAXS_CUDA(cudaMemcpyAsync(base + off_mb, &mbv, 4, cudaMemcpyHostToDevice, s));
    AUSAXS_CUDA(cudaMemcpyAsync(base + off_q, q, (size_t)nq * 8, cudaMemcpyHostToDevice, s));
    HostDebye out;
    DebyeArgs& A = out.A;
    A = DebyeArgs{};
    A.R = R;
    A.nb = mb;
    A.H = reinterpret_cast<const double*>(base + off_H);
    A.axis0 = reinterpret_cast<const double*>(base + off_ax0);
    A.axis1 = grid ? reinterpret_cast<const double*>(base + off_ax1) : A.axis0;
    A.axis2 = grid ? reinterpret_cast<const double*>(base + off_ax2) : A.axis0;
    A.max_bin = reinterpret_cast<const int32_t*>(base + off_mb);
    A.rows = reinterpret_cast<const RowDesc*>(base + off_rows);
    A.overflow = nullptr;
    A.exv_model = grid ? 1 : (cfg.manager == AUSAXS_MANAGER_FFEXPLICIT ? 2 : 0);
    A.cw = p.cw;
    A.cx = p.cx;
    A.crho = p.crho;
    A.dw_atomic = p.dw_atomic;
    A.dw_exv = p.dw_exv;
    A.grid_volume = p.grid_width * p.grid_width * p.grid_width;
    A.q = reinterpret_cast<const double*>(base + off_q);
    A.nq = nq;
    A.tolerance = p.tolerance > 0 ? p.tolerance : 1e-5;
    A.Iq = reinterpret_cast<double*>(base + off_I);
    A.profiles = reinterpret_cast<double*>(base + off_P);
    int32_t* cols = reinterpret_cast<int32_t*>(base + off_mb) + 1;
    AUSAXS_CUDA(cudaMemsetAsync(cols, 0, 4, s));
    A.fp64_columns = cols;
    A.tc_err_est = p.precision != 1 ? reinterpret_cast<double*>(base + off_E) : nullptr;
    out.extra = base + off_X;
    out.groups = grid ? 7 : 1;
    return out;
}

void debye_of_host_histogram(Ctx& C, const ausaxs_hist_config& cfg, const ausaxs_hist_result& h, const double* q,
                             int nq, const ausaxs_debye_params& p, double* Iq, double* profiles) {
    HostDebye D = upload_host_histogram(C, cfg, h, q, nq, p, 0);
    DebyeArgs& A = D.A;
    double* prof_dev = A.profiles;
    if (!profiles) A.profiles = nullptr;
    cudaStream_t s = C.stream;
    C.last_tc_err.assign(p.precision != 1 ? nq : 0, INFINITY);
    if (nq > 0) {
        const int used = run_debye(C, A, D.groups, C.tc, p.precision, &C.x, cfg.bin_width);
        int32_t ncols = 0;
        AUSAXS_CUDA(cudaMemcpyAsync(&ncols, A.fp64_columns, 4, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaMemcpyAsync(Iq, A.Iq, (size_t)nq * 8, cudaMemcpyDeviceToHost, s));
        if (profiles) AUSAXS_CUDA(cudaMemcpyAsync(profiles, prof_dev, (size_t)nq * 6 * 8, cudaMemcpyDeviceToHost, s));
        if (p.precision != 1)
            AUSAXS_CUDA(cudaMemcpyAsync(C.last_tc_err.data(), A.tc_err_est, (size_t)nq * 8, cudaMemcpyDeviceToHost, s));
        AUSAXS_CUDA(cudaStreamSynchronize(s));
        C.last_fp64_columns = (used == 0 || used == 3) ? ncols : nq;
    }
    AUSAXS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace ausaxs_b200
