// Host-side engine: device-resident structures and the launch plans of the Debye hot path.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/ausaxs_b200.h"
#include "debye.cuh"
#include "finalize.cuh"
#include "lattice.cuh"
#include "pairhist.cuh"
#include "prep.cuh"

namespace ausaxs_b200 {

// Error raised inside the engine; the C ABI turns it into a status code plus last-error text.
struct Error {
    int code;
    std::string msg;
};

#define AUSAXS_CUDA(call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) throw ::ausaxs_b200::Error{AUSAXS_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)}; \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// A growable device allocation (grows, never shrinks; freed with its owner).
struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    bool owned = true;  // false: a view into memory owned elsewhere (never grown or freed here)
    void ensure(size_t bytes);
    void view(void* ptr, size_t bytes) {
        p = ptr;
        n = bytes;
        owned = false;
    }
    ~DevBuf();
    template <typename T>
    T* as(size_t byte_offset = 0) const { return reinterpret_cast<T*>(static_cast<char*>(p) + byte_offset); }
};

struct Ctx;

// One pass of pair binning of a structure before it is cut into tiles: the two point sets, the
// rows it increments, and where its global accumulators live.
struct JobSpec {
    const float4* A;
    int na;
    const float4* B;
    int nbp;
    int self, rmode, rows;
    unsigned long long* counts;  // [rows][nb]
    unsigned long long* dsum;    // [nb] or null
    long long* wsum;             // [nb] or null
    // scalar-tail geometry (PairJob): -1 = a plain job (tail_end = nbp, tail_from_outer = self)
    int a_base = 0, b_base = 0, tail_end = -1, tail_from_outer = -1;
    int mult = 1;  // multiplicity of every pair (PairJob::mult)
    bool lattice = false;  // the plan bins this pass with the lattice kernel (the structure's own launches)
};

// Buffers of the exact-accumulation tensor-core transform of one structure's rows (debye_x.cu), kept
// with their shape so repeated transforms reuse tables, digit blocks and planes.
struct XBufs {
    DevBuf table, cpart, qcache, flags, planes, rows, adig, tile_off, row_scale;
    XPlan plan{};
    // shape the buffers were made for
    const double* H = nullptr;
    const double* q = nullptr;
    int R = 0, nb = 0, nq = 0;
    double w = 0, qmax = -1;
};

// Launch plan of one structure under one histogram configuration: job table, accumulator and
// output layout, kernel shapes.  Built once, then enqueued any number of times without
// allocation or synchronisation (so it can be captured in a CUDA graph).
struct Plan {
    // key
    int manager = 0, weighted = 0, bin_count = 0;
    double bin_width = 0;
    int n_a = -1, n_w = -1, n_x = -1, T = -1;
    // shapes
    int nb = 0, tile = 256;
    struct Group {  // one pair-kernel launch
        PairLaunch launch{};
        int tile = 256, grid = 0;
        size_t smem = 0;
    } group[3];
    int n_launch = 0;
    long long total_tiles = 0, pairs = 0;
    int R = 0;
    float inv_w = 0, c = 0, scale = 0;
    // device layout
    DevBuf dev;
    size_t off_jobs = 0, off_acc = 0, acc_bytes = 0, off_counter = 0, off_overflow = 0, off_maxbin = 0, off_wscale = 0,
           off_self = 0, off_fp64cols = 0, off_H = 0, off_tot = 0, off_d = 0, off_dax = 0, off_dxx = 0, off_rows = 0,
           off_expand_aa = 0, off_expand_aw = 0;  // in `expand`, allocated by the first host read-back
    DevBuf expand;
    FinalizeFF fin_ff{};
    FinalizeMT fin_mt{};
    std::vector<JobSpec> specs;  // the structure's passes (tiled by append_pair_jobs)
    std::vector<RowDesc> rows_host;  // the Debye rows (device copy at off_rows)
    int max_group_rows = 1;      // rows that fit on chip at once (for 512-point tiles)
    // tensor-core scratch
    DevBuf tc;
    int tc_nq = 0;
    XBufs x;
    // the dummies' self pairs by the lattice kernel (lattice.cuh): launch shape, or grid == 0
    LatticeLaunch lattice{};
    int lattice_grid = 0;
    size_t lattice_smem = 0;
};

// Lattice form of a structure's excluded-volume dummies, built on the first plan that asks for it.
struct StructureLattice {
    bool tried = false;   // built (or found unusable) already
    bool usable = false;  // integer coordinates, no shared cells, lines short enough
    LatticeGrid G;
    long long s2_max = 0;  // largest squared offset between two dummies
    DevBuf lines, table, scratch;
};

struct Structure {
    Ctx* ctx = nullptr;
    int ff_typed = 0;
    int n_a = 0, n_w = 0, n_x = 0;
    DevBuf raw_a, raw_w, raw_x, dense_a, meta;
    int T = 0;
    int type_ff[kNff] = {};
    int type_count[kNff] = {};
    int ff_to_type[kNff] = {};
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    float dmax = 0;
    float dmax_extra = 0;  // distance range kept beyond the current bounding-box diagonal (moving bodies)
    Plan plan;
    StructureLattice lat;
    // the dummies on the integer lattice (synchronises once per structure); true when usable
    bool lattice_ready();

    // copy in (host or device pointers), census, validation and dense-type conversion (one sync)
    void load(const float* atoms, int n_atoms, const float* waters, int n_waters, const float* exv, int n_exv,
              int ff_typed_, bool host, int exv_host = -1);
    // (exv_host: where exv lives when it differs from the other arrays; -1 = as `host`)
    // the same in two halves, so many structures share one synchronisation: load_begin enqueues the
    // copies and the census into d_stats and its read-back into h_stats (pinned); after the stream has
    // been synchronised, load_end validates and enqueues the dense-type conversion
    void load_begin(const float* atoms, int n_atoms, const float* waters, int n_waters, const float* exv, int n_exv,
                    int ff_typed_, bool host, PrepStats* h_stats, PrepStats* d_stats, int exv_host = -1);
    void load_end(const PrepStats& st);
    int32_t hmeta[2 * kNff] = {};  // host copy of meta (type counts, ff -> dense type)
    const float4* atoms_for_pairs() const { return ff_typed ? dense_a.as<float4>() : raw_a.as<float4>(); }
    Plan& plan_for(const ausaxs_hist_config& cfg);
    void enqueue_histogram(const ausaxs_hist_config& cfg);
    void enqueue_debye(const ausaxs_hist_config& cfg, const double* q_dev, int nq, const ausaxs_debye_params& p,
                       double* Iq_dev, double* prof_dev);
    // arguments of the FP64 transform of the planned histogram (no launch)
    DebyeArgs debye_args(const ausaxs_hist_config& cfg, const double* q_dev, int nq, const ausaxs_debye_params& p,
                         double* Iq_dev, double* prof_dev);
    // histogram in the reference's layouts into host buffers (synchronises)
    void read_histogram(const ausaxs_hist_config& cfg, ausaxs_hist_result* out);
};

struct GridExv;
struct Hydrator;

struct Ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    long long launches = 0;
    // optional per-kernel-class timing with CUDA events on the context's stream
    // (class 0: pair histograms, 1: finalisation, 2: FP64 Debye transform, 3: tensor-core Debye transform,
    // 4: grid excluded volume, 5: hydration, 6: lattice pairs of grid dummies)
    bool timing = false;
    struct Timed {
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
        double ms = 0;
        long long count = 0;
    } timed[7];
    void time_begin(int cls, cudaEvent_t* ev);
    void time_end(int cls, cudaEvent_t ev);
    void time_collect();
    DevBuf stats;
    PrepStats* h_stats = nullptr;  // pinned
    PrepStats* h_stats_many = nullptr;  // pinned, census slots of batched loads (grows, freed with the context)
    size_t n_stats_many = 0;
    PrepStats* stats_slots(size_t n);
    std::unique_ptr<Structure> scratch;
    std::shared_ptr<GridExv> grid;  // molecular-grid workspace of one-shot calls (gridexv.cuh)
    std::shared_ptr<Hydrator> hyd;  // hydration workspace (hydrate.cuh)
    DevBuf io;                     // q / I(q) / profiles of one-shot host calls
    DevBuf tc;                     // tensor-core scratch of one-shot host calls
    XBufs x;                       // exact tensor-core transform of one-shot host calls
    int last_fp64_columns = 0;     // q values the last host transform evaluated in FP64
    std::vector<double> last_tc_err;  // per q: estimated relative error of its tensor-core value
    void check_launch(const char* what);
};

// Cuts the passes of a planned structure into tiles of `tile` points and appends them to launch
// classes: 0 (one on-chip row), 1 (up to T rows), 2 (more), or all to class 0 when !by_class.
// Tile ids continue from tiles[g]; rows[g] grows to the largest row group of class g.  Row groups
// hold at most max_rows rows (0: the plan's own limit).
// skip_lattice: leave out the passes the plan bins with the lattice kernel.
void append_pair_jobs(const Plan& P, int tile, bool by_class, std::vector<PairJob> (&jobs)[3], long long (&tiles)[3],
                      int (&rows)[3], int max_rows = 0, bool skip_lattice = false);

// Clears n device ranges of u64 words in one launch (table in device memory); a range with a
// source is set to the source's words instead.
struct ZeroRange {
    unsigned long long* p;
    long long words;
    const unsigned long long* src = nullptr;
};
void zero_ranges_launch(const ZeroRange* ranges_dev, int n, cudaStream_t s);

// Split-BF16 tensor-core contraction (precision 0) or exact-accumulation tensor-core contraction
// (precision 3, needs xb and the bin width w) followed by the FP64 epilogue, or FP64 only (precision
// 1); precision 2 picks 3 when the contraction pays off (debye_precision), else 1.  Returns the
// precision used.
int run_debye(Ctx& C, DebyeArgs& A, int groups_present, DevBuf& tc, int precision, XBufs* xb = nullptr,
              double w = 0);

// The contraction's fixed cost (operand staging in a few CTAs, ~50 us) exceeds the FP64 transform's
// below about 5e6 row x bin x q products (measured: 48 us against 25 us at 2.4e6, 92 + ~50 us
// against ~400 us at 5.4e7); precision 2 uses the tensor cores from 8e6 on.
constexpr double kTcMinWork = 8e6;
inline int debye_precision(int precision, int rows, int bins, int nq) {
    if (precision != 2) return precision;
    return (double)rows * bins * nq >= kTcMinWork ? 3 : 1;
}

// A histogram given in the reference's host layouts (ausaxs_hist_result), compacted to the rows of
// the form-factor types present and uploaded into the context's io buffer with q: the transform's
// arguments (I(q) and profiles [6][nq] in the io buffer too) and extra_bytes of scratch after them.
struct HostDebye {
    DebyeArgs A;
    char* extra = nullptr;
    int groups = 1;  // distance-axis groups present (run_debye)
};
HostDebye upload_host_histogram(Ctx& C, const ausaxs_hist_config& cfg, const ausaxs_hist_result& h, const double* q,
                                int nq, const ausaxs_debye_params& p, size_t extra_bytes);

// CompositeDistanceHistogram*::debye_transform() of a host histogram (synchronises).
void debye_of_host_histogram(Ctx& C, const ausaxs_hist_config& cfg, const ausaxs_hist_result& h, const double* q,
                             int nq, const ausaxs_debye_params& p, double* Iq, double* profiles);

}  // namespace ausaxs_b200

struct ausaxs_gpu_ctx {
    ausaxs_b200::Ctx impl;
};

struct ausaxs_gpu_structure {
    ausaxs_b200::Structure impl;
};
