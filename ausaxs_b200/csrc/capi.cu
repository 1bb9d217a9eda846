// The C ABI (include/ausaxs_b200.h): status codes and last-error text instead of exceptions, the
// convention of the reference's own C API (include/api/api/api_helper.h:15-45).
#include <cmath>
#include <cstring>
#include <string>

#include "engine.cuh"
#include "fit.cuh"
#include "gridexv.cuh"
#include "hydrate.cuh"
#include "guard.cuh"
#include "lsq.cuh"

using namespace ausaxs_b200;

namespace {
thread_local std::string g_last_error;

Structure& scratch(Ctx& C) {
    if (!C.scratch) {
        C.scratch = std::make_unique<Structure>();
        C.scratch->ctx = &C;
    }
    return *C.scratch;
}

GridExv& grid_workspace(Ctx& C) {
    if (!C.grid) C.grid = std::make_shared<GridExv>();
    return *C.grid;
}

bool ff_manager(int m) { return m == AUSAXS_MANAGER_FFAVG || m == AUSAXS_MANAGER_FFEXPLICIT || m == AUSAXS_MANAGER_FFGRID; }

void check_cfg(const ausaxs_hist_config* cfg) {
    if (!cfg) throw Error{AUSAXS_ERR_ARGUMENT, "null configuration"};
}

// Loads an FF-typed structure and runs its molecular grid (RawGridExv on the expanded grid); with
// with_dummies the structure is reloaded with the grid's dummies as its excluded-volume points.
// Returns the grid volume (Molecule::get_volume_grid()).
double load_with_grid(Structure& S, const float* atoms, int32_t n_atoms, const float* waters, int32_t n_waters,
                      bool host, bool with_dummies) {
    Ctx& C = *S.ctx;
    S.load(atoms, n_atoms, waters, n_waters, nullptr, 0, 1, host);  // census: validation and bounding box
    GridExv& g = grid_workspace(C);
    g.run(C, S.raw_a.as<float4>(), n_atoms, S.raw_w.as<float4>(), n_waters, S.lo, S.hi, with_dummies);
    if (with_dummies) S.load(atoms, n_atoms, waters, n_waters, g.points.as<float>(), (int)g.count, 1, host, 0);
    return g.volume;
}

// The scratch structure of a one-shot host call, with the grid-derived inputs the configuration asks
// for: FFGRID with n_exv = AUSAXS_EXV_FROM_GRID takes its dummies from the molecular grid (RawGridExv,
// generated on the device), FFAVG with z_exv < 0 takes Z_exv = V_grid rho_w / N_atoms from the grid
// volume (HistogramManagerMTFFAvg.cpp:351-364 with Molecule::get_volume_grid()).  Returns the effective
// configuration.
ausaxs_hist_config load_scratch(Ctx& C, const ausaxs_hist_config& cfg, const float* atoms, int32_t n_atoms,
                                const float* waters, int32_t n_waters, const float* exv, int32_t n_exv) {
    Structure& S = scratch(C);
    ausaxs_hist_config c = cfg;
    const bool grid = cfg.manager == AUSAXS_MANAGER_FFGRID;
    const bool gen = grid && n_exv == AUSAXS_EXV_FROM_GRID;
    const bool zgrid = cfg.manager == AUSAXS_MANAGER_FFAVG && cfg.z_exv < 0;
    if (!gen && !zgrid) {
        if (n_exv < 0 && grid) throw Error{AUSAXS_ERR_ARGUMENT, "negative exv count"};
        S.load(atoms, n_atoms, waters, n_waters, grid ? exv : nullptr, grid ? n_exv : 0, ff_manager(cfg.manager), true);
        return c;
    }
    const double volume = load_with_grid(S, atoms, n_atoms, waters, n_waters, true, gen);
    if (zgrid) c.z_exv = n_atoms ? volume * 0.334 / n_atoms : 0.0;  // rho_w (Constants.h:114)
    return c;
}

ausaxs_debye_params default_params(const ausaxs_debye_params* p) {
    if (p) return *p;
    ausaxs_debye_params d{};
    d.cw = d.cx = d.crho = 1.0;
    d.grid_width = 1.0;
    d.precision = 0;
    d.tolerance = 1e-5;
    return d;
}
// The search of a fit: interval, Golden constants and iteration count as mini::Golden forms them
// (Golden.h:36-37, Golden.cpp:26-46); limits per parameter from ICompositeDistanceHistogram.h:70 and
// ICompositeDistanceHistogramExv.cpp:8-12.
FitArgs fit_search(const ausaxs_hist_config& cfg, const ausaxs_fit_options* o, const ausaxs_debye_params& base) {
    if (!o || o->parameter < 0 || o->parameter > 4) throw Error{AUSAXS_ERR_ARGUMENT, "fit parameter must be 0..4"};
    const bool mt = cfg.manager == AUSAXS_MANAGER_MT;
    if (mt && o->parameter != 0) throw Error{AUSAXS_ERR_ARGUMENT, "the Simple histogram has the water scaling only"};
    static const double limits[5][2] = {{0.0, 10.0}, {0.92, 1.08}, {0.5, 2.0}, {0.0, 5.0}, {0.0, 5.0}};
    FitArgs F{};
    F.model = mt ? kFitSimple : (cfg.manager == AUSAXS_MANAGER_FFEXPLICIT ? kFitExplicitExv : kFitAverageExv);
    F.param = o->parameter;
    F.lo = o->lo == o->hi ? limits[o->parameter][0] : o->lo;
    F.hi = o->lo == o->hi ? limits[o->parameter][1] : o->hi;
    if (!(std::isfinite(F.lo) && std::isfinite(F.hi))) throw Error{AUSAXS_ERR_ARGUMENT, "non-finite search interval"};
    const double tol = o->tolerance > 0 ? o->tolerance : 1e-4;
    const double phi = (1 + std::sqrt(5.0)) / 2;
    F.invphi = 1 / phi;
    F.invphi2 = F.invphi * F.invphi;
    double a = F.lo, b = F.hi;
    const double temp = a + b;
    a = std::min(a, b);
    b = temp - a;
    const double diff = b - a;
    F.steps = diff < tol ? -1 : (int)std::ceil(std::log(tol / diff) / std::log(F.invphi));
    F.base[0] = base.cw;
    F.base[1] = base.cx;
    F.base[2] = base.crho;
    F.base[3] = base.dw_atomic;
    F.base[4] = base.dw_exv;
    return F;
}

// The transform parameters of the unit profiles: cw = cx = crho = 1, no Debye-Waller factors, FP64.
ausaxs_debye_params unit_params(const ausaxs_debye_params& base) {
    ausaxs_debye_params u = base;
    u.cw = u.cx = u.crho = 1.0;
    u.dw_atomic = u.dw_exv = 0.0;
    u.precision = 1;
    return u;
}

void read_fit(Ctx& C, const double* out_dev, ausaxs_fit_result* out) {
    double o[7];
    AUSAXS_CUDA(cudaMemcpyAsync(o, out_dev, sizeof o, cudaMemcpyDeviceToHost, C.stream));
    AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    out->value = o[0];
    out->a = o[1];
    out->b = o[2];
    out->chi2 = o[3];
    out->evaluations = (int32_t)o[4];
    out->a_err = o[5];
    out->b_err = o[6];
}
}  // namespace

namespace ausaxs_b200 {
// Lets entry points outside this file report through ausaxs_gpu_last_error().
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace ausaxs_b200

struct ausaxs_gpu_hydration_grid {
    ausaxs_gpu_ctx* ctx = nullptr;
    double gmin[3] = {0, 0, 0};
    int bins[3] = {0, 0, 0};
    DevBuf cells;  // cell states, then an error word
    DevBuf stage;  // atoms and types of add / remove calls
    size_t cell_bytes = 0;
};

namespace {
// form-factor types with a radius (get_vdw_radius(form_factor_t) throws for EXCLUDED_VOLUME, COUNT and
// unknown values), finite coordinates, and (axes given) every atom's cell inside the grid
void check_hydration_atoms(const double* atoms, const int32_t* ff, int64_t n, const double* gmin, const int* bins) {
    for (int64_t a = 0; a < n; ++a) {
        const int32_t f = ff[a];
        if (f < 1 || f > 16 || f == 15) throw Error{AUSAXS_ERR_FORM_FACTOR, "form-factor type without a radius"};
        for (int d = 0; d < 3; ++d) {
            if (!std::isfinite(atoms[3 * a + d])) throw Error{AUSAXS_ERR_ARGUMENT, "non-finite atom coordinate"};
            if (gmin) {
                const double b = std::round(atoms[3 * a + d] - gmin[d]);
                if (!(b >= 0 && b < bins[d])) throw Error{AUSAXS_ERR_ARGUMENT, "an atom lies outside the hydration grid"};
            }
        }
    }
}

void read_axes(const double* axes, double gmin[3], int bins[3]) {
    for (int d = 0; d < 3; ++d) {
        gmin[d] = axes[d];
        bins[d] = (int)axes[3 + d];
        if (!std::isfinite(axes[d]) || !(axes[3 + d] >= 1 && axes[3 + d] < 2147483647.0) || axes[3 + d] != (double)bins[d])
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid hydration grid axes"};
    }
    hydration_cells_check(gmin, bins);
}

Hydrator& hydrator(Ctx& C) {
    if (!C.hyd) C.hyd = std::make_shared<Hydrator>();
    return *C.hyd;
}

// atoms, types and noise into the hydrator's input buffer
void stage_hydration_inputs(Ctx& C, Hydrator& H, const double* atoms, const int32_t* ff, int64_t n, const double* noise,
                            double** d_atoms, int32_t** d_ff, double** d_noise) {
    const size_t a_bytes = align_up((size_t)n * 24, 256), f_bytes = align_up((size_t)n * 4, 256);
    const size_t n_bytes = noise ? (size_t)n * AUSAXS_HYDRATE_DIRECTIONS * 24 : 0;
    H.in.ensure(a_bytes + f_bytes + n_bytes + 256);
    *d_atoms = H.in.as<double>();
    *d_ff = H.in.as<int32_t>(a_bytes);
    *d_noise = noise ? H.in.as<double>(a_bytes + f_bytes) : nullptr;
    if (n) {
        AUSAXS_CUDA(cudaMemcpyAsync(*d_atoms, atoms, (size_t)n * 24, cudaMemcpyHostToDevice, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(*d_ff, ff, (size_t)n * 4, cudaMemcpyHostToDevice, C.stream));
        if (noise) AUSAXS_CUDA(cudaMemcpyAsync(*d_noise, noise, n_bytes, cudaMemcpyHostToDevice, C.stream));
    }
}

void read_waters(Ctx& C, Hydrator& H, double* waters_out, int64_t capacity, int64_t* n_waters, int64_t* candidates_out,
                 int32_t* rounds) {
    *n_waters = H.count;
    if (rounds) *rounds = H.rounds;
    if (capacity > 0 && H.count > 0) {
        if (capacity < H.count) throw Error{AUSAXS_ERR_CAPACITY, "waters_out holds fewer waters than were placed"};
        AUSAXS_CUDA(cudaMemcpyAsync(waters_out, H.waters(), (size_t)H.count * 24, cudaMemcpyDeviceToHost, C.stream));
        if (candidates_out)
            AUSAXS_CUDA(cudaMemcpyAsync(candidates_out, H.candidates(), (size_t)H.count * 8, cudaMemcpyDeviceToHost, C.stream));
    }
    AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
}

bool bad_hydrate_args(const double* atoms, const int32_t* ff, int64_t n, double* waters_out, int64_t capacity,
                      int64_t* n_waters) {
    return !n_waters || n < 0 || (n && (!atoms || !ff)) || capacity < 0 || (capacity > 0 && !waters_out);
}
}  // namespace

namespace {
int hydration_grid_edit(ausaxs_gpu_hydration_grid* g, const double* atoms, const int32_t* ff, int64_t n, bool add) {
    return guarded([&] {
        if (!g || n < 0 || (n && (!atoms || !ff))) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        check_hydration_atoms(atoms, ff, n, g->gmin, g->bins);
        if (!n) return;
        Ctx& C = g->ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const size_t a_bytes = align_up((size_t)n * 24, 256);
        g->stage.ensure(a_bytes + align_up((size_t)n * 4, 256));
        double* d_atoms = g->stage.as<double>();
        int32_t* d_ff = g->stage.as<int32_t>(a_bytes);
        AUSAXS_CUDA(cudaMemcpyAsync(d_atoms, atoms, (size_t)n * 24, cudaMemcpyHostToDevice, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(d_ff, ff, (size_t)n * 4, cudaMemcpyHostToDevice, C.stream));
        int* err = g->cells.as<int>(g->cell_bytes);
        if (add) hydration_add(C, g->cells.as<uint8_t>(), g->gmin, g->bins, d_atoms, d_ff, n, err);
        else hydration_remove(C, g->cells.as<uint8_t>(), g->gmin, g->bins, d_atoms, d_ff, n, err);
        // the staging buffer is reused by the next call: let this one finish with it
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    });
}
}  // namespace

extern "C" {

const char* ausaxs_gpu_last_error(void) { return g_last_error.c_str(); }

int ausaxs_gpu_ctx_create(int device, ausaxs_gpu_ctx** out) {
    return guarded([&] {
        if (!out) throw Error{AUSAXS_ERR_ARGUMENT, "null output"};
        *out = nullptr;
        int n = 0;
        AUSAXS_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw Error{AUSAXS_ERR_ARGUMENT, "no such CUDA device"};
        AUSAXS_CUDA(cudaSetDevice(device));
        auto* c = new ausaxs_gpu_ctx();
        Ctx& C = c->impl;
        C.device = device;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) C.sm_count = prop.multiProcessorCount;
        if (cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete c;
            throw Error{AUSAXS_ERR_CUDA, "cudaStreamCreate failed"};
        }
        C.own_stream = true;
        if (cudaMallocHost(&C.h_stats, sizeof(PrepStats)) != cudaSuccess) {
            cudaStreamDestroy(C.stream);
            delete c;
            throw Error{AUSAXS_ERR_CUDA, "cudaMallocHost failed"};
        }
        *out = c;
    });
}

int ausaxs_gpu_ctx_destroy(ausaxs_gpu_ctx* ctx) {
    return guarded([&] {
        if (!ctx) return;
        Ctx& C = ctx->impl;
        cudaSetDevice(C.device);
        cudaStreamSynchronize(C.stream);
        C.scratch.reset();
        if (C.h_stats) cudaFreeHost(C.h_stats);
        if (C.h_stats_many) cudaFreeHost(C.h_stats_many);
        if (C.own_stream) cudaStreamDestroy(C.stream);
        delete ctx;
    });
}

int ausaxs_gpu_ctx_set_stream(ausaxs_gpu_ctx* ctx, void* stream) {
    return guarded([&] {
        if (!ctx) throw Error{AUSAXS_ERR_ARGUMENT, "null context"};
        Ctx& C = ctx->impl;
        if (C.own_stream) {
            cudaStreamSynchronize(C.stream);
            cudaStreamDestroy(C.stream);
            C.own_stream = false;
        }
        if (stream) {
            C.stream = static_cast<cudaStream_t>(stream);
        } else {
            AUSAXS_CUDA(cudaStreamCreateWithFlags(&C.stream, cudaStreamNonBlocking));
            C.own_stream = true;
        }
    });
}

int64_t ausaxs_gpu_ctx_launch_count(const ausaxs_gpu_ctx* ctx) { return ctx ? ctx->impl.launches : 0; }

int ausaxs_gpu_ctx_enable_timing(ausaxs_gpu_ctx* ctx, int32_t enable) {
    return guarded([&] {
        if (!ctx) throw Error{AUSAXS_ERR_ARGUMENT, "null context"};
        Ctx& C = ctx->impl;
        C.time_collect();
        for (auto& t : C.timed) t.ms = 0, t.count = 0;
        C.timing = enable != 0;
    });
}

int ausaxs_gpu_ctx_kernel_time(ausaxs_gpu_ctx* ctx, int32_t kernel_class, double* ms, int64_t* launches) {
    return guarded([&] {
        if (!ctx || kernel_class < 0 || kernel_class > 6) throw Error{AUSAXS_ERR_ARGUMENT, "bad argument"};
        Ctx& C = ctx->impl;
        C.time_collect();
        if (ms) *ms = C.timed[kernel_class].ms;
        if (launches) *launches = C.timed[kernel_class].count;
    });
}

int ausaxs_gpu_ctx_fp64_columns(ausaxs_gpu_ctx* ctx, int32_t* n) {
    return guarded([&] {
        if (!ctx || !n) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        *n = ctx->impl.last_fp64_columns;
    });
}

int ausaxs_gpu_ctx_tc_error_estimate(ausaxs_gpu_ctx* ctx, double* out, int32_t nq) {
    return guarded([&] {
        if (!ctx || (nq > 0 && !out)) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        const auto& e = ctx->impl.last_tc_err;
        if ((size_t)nq != e.size()) throw Error{AUSAXS_ERR_ARGUMENT, "nq differs from the last tensor-core transform"};
        std::copy(e.begin(), e.end(), out);
    });
}

int ausaxs_gpu_histogram(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const float* atoms, int32_t n_atoms,
                         const float* waters, int32_t n_waters, const float* exv, int32_t n_exv,
                         ausaxs_hist_result* out) {
    return guarded([&] {
        if (!ctx || !out) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        check_cfg(cfg);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const ausaxs_hist_config c = load_scratch(C, *cfg, atoms, n_atoms, waters, n_waters, exv, n_exv);
        Structure& S = scratch(C);
        S.enqueue_histogram(c);
        S.read_histogram(c, out);
    });
}

int ausaxs_gpu_debye(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const ausaxs_hist_result* hist,
                     const double* q, int32_t n_q, const ausaxs_debye_params* params, double* Iq, double* profiles) {
    return guarded([&] {
        if (!ctx || !hist || !q || !Iq || n_q < 0) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        check_cfg(cfg);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        ausaxs_debye_params p = default_params(params);
        debye_of_host_histogram(C, *cfg, *hist, q, n_q, p, Iq, profiles);
    });
}

int ausaxs_gpu_profile(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const float* atoms, int32_t n_atoms,
                       const float* waters, int32_t n_waters, const float* exv, int32_t n_exv, const double* q,
                       int32_t n_q, const ausaxs_debye_params* params, double* Iq, double* profiles) {
    return guarded([&] {
        if (!ctx || !q || !Iq || n_q < 0) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        check_cfg(cfg);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const ausaxs_hist_config c = load_scratch(C, *cfg, atoms, n_atoms, waters, n_waters, exv, n_exv);
        Structure& S = scratch(C);
        ausaxs_debye_params p = default_params(params);
        size_t need = (size_t)n_q * 8 * 8 + 256;
        C.io.ensure(need);
        double* dq = C.io.as<double>();
        double* dI = dq + n_q;
        double* dP = dI + n_q;
        AUSAXS_CUDA(cudaMemcpyAsync(dq, q, (size_t)n_q * 8, cudaMemcpyHostToDevice, C.stream));
        S.enqueue_histogram(c);
        S.enqueue_debye(c, dq, n_q, p, dI, profiles ? dP : nullptr);
        AUSAXS_CUDA(cudaMemcpyAsync(Iq, dI, (size_t)n_q * 8, cudaMemcpyDeviceToHost, C.stream));
        if (profiles) AUSAXS_CUDA(cudaMemcpyAsync(profiles, dP, (size_t)n_q * 6 * 8, cudaMemcpyDeviceToHost, C.stream));
        unsigned long long overflow = 0;
        AUSAXS_CUDA(cudaMemcpyAsync(&overflow, S.plan.dev.as<char>() + S.plan.off_overflow, 8, cudaMemcpyDeviceToHost, C.stream));
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
        if (overflow) throw Error{AUSAXS_ERR_BIN_OVERFLOW, "pair distances beyond bin_count * bin_width; increase settings::axes::bin_count"};
    });
}

int ausaxs_gpu_linear_lsq(ausaxs_gpu_ctx* ctx, const double* data, const double* model, const double* err,
                          int32_t n, double* out) {
    return guarded([&] {
        if (!ctx || !data || !model || !err || !out || n < 2) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        C.io.ensure((size_t)n * 3 * 8 + 256);
        double* d = C.io.as<double>();
        AUSAXS_CUDA(cudaMemcpyAsync(d, data, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(d + n, model, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(d + 2 * n, err, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
        double* o = d + 3 * (size_t)n;
        lsq_launch(d, d + n, d + 2 * n, n, o, C.stream);
        C.check_launch("lsq");
        AUSAXS_CUDA(cudaMemcpyAsync(out, o, 5 * 8, cudaMemcpyDeviceToHost, C.stream));
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ausaxs_gpu_structure_create(ausaxs_gpu_ctx* ctx, int32_t ff_typed, const float* atoms, int32_t n_atoms,
                                const float* waters, int32_t n_waters, const float* exv, int32_t n_exv,
                                int32_t host_pointers, ausaxs_gpu_structure** out) {
    return guarded([&] {
        if (!ctx || !out) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        *out = nullptr;
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        auto* h = new ausaxs_gpu_structure();
        h->impl.ctx = &C;
        try {
            if (n_exv == AUSAXS_EXV_FROM_GRID) {
                if (!ff_typed) throw Error{AUSAXS_ERR_ARGUMENT, "grid excluded volume needs form-factor typed atoms"};
                load_with_grid(h->impl, atoms, n_atoms, waters, n_waters, host_pointers != 0, true);
            } else {
                h->impl.load(atoms, n_atoms, waters, n_waters, exv, n_exv, ff_typed ? 1 : 0, host_pointers != 0);
            }
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int ausaxs_gpu_structure_destroy(ausaxs_gpu_structure* s) {
    return guarded([&] {
        if (!s) return;
        cudaStreamSynchronize(s->impl.ctx->stream);
        delete s;
    });
}

int ausaxs_gpu_structure_profile(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                                 const double* q, int32_t n_q, const ausaxs_debye_params* params, double* Iq,
                                 double* profiles) {
    return guarded([&] {
        if (!ctx || !s || !q || !Iq || n_q < 0) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        check_cfg(cfg);
        if (s->impl.ctx != &ctx->impl) throw Error{AUSAXS_ERR_ARGUMENT, "structure belongs to another context"};
        ausaxs_debye_params p = default_params(params);
        s->impl.enqueue_histogram(*cfg);
        s->impl.enqueue_debye(*cfg, q, n_q, p, Iq, profiles);
    });
}

int ausaxs_gpu_structure_histogram(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                                   ausaxs_hist_result* out) {
    return guarded([&] {
        if (!ctx || !s || !out) throw Error{AUSAXS_ERR_ARGUMENT, "null argument"};
        check_cfg(cfg);
        s->impl.enqueue_histogram(*cfg);
        s->impl.read_histogram(*cfg, out);
    });
}

int ausaxs_gpu_fit(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const ausaxs_hist_result* hist, const double* q,
                   const double* I, const double* sigma, int32_t n, const ausaxs_debye_params* base,
                   const ausaxs_fit_options* options, ausaxs_fit_result* out, double* I_fit) {
    return guarded([&] {
        if (!ctx || !hist || !q || !I || !sigma || !out || n < 2) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        check_cfg(cfg);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const ausaxs_debye_params b = default_params(base);
        FitArgs F = fit_search(*cfg, options, b);
        const size_t vec = align_up((size_t)n * 8, 256);
        HostDebye D = upload_host_histogram(C, *cfg, *hist, q, n, unit_params(b), 5 * vec + 256);
        double* y = reinterpret_cast<double*>(D.extra);
        double* sg = reinterpret_cast<double*>(D.extra + vec);
        F.Iw = reinterpret_cast<double*>(D.extra + 2 * vec);
        F.I_fit = I_fit ? reinterpret_cast<double*>(D.extra + 3 * vec) : nullptr;
        F.W = reinterpret_cast<double*>(D.extra + 4 * vec);
        F.out = reinterpret_cast<double*>(D.extra + 5 * vec);
        AUSAXS_CUDA(cudaMemcpyAsync(y, I, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
        AUSAXS_CUDA(cudaMemcpyAsync(sg, sigma, (size_t)n * 8, cudaMemcpyHostToDevice, C.stream));
        run_debye(C, D.A, D.groups, C.tc, 1);
        F.nq = n;
        F.q = D.A.q;
        F.P = D.A.profiles;
        F.y = y;
        F.sigma = sg;
        fit_launch(F, C.stream);
        C.check_launch("fit");
        if (I_fit) AUSAXS_CUDA(cudaMemcpyAsync(I_fit, F.I_fit, (size_t)n * 8, cudaMemcpyDeviceToHost, C.stream));
        read_fit(C, F.out, out);
    });
}

int ausaxs_gpu_structure_fit(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                             const double* q, const double* I, const double* sigma, int32_t n,
                             const ausaxs_debye_params* base, const ausaxs_fit_options* options, ausaxs_fit_result* out,
                             double* I_fit) {
    return guarded([&] {
        if (!ctx || !s || !q || !I || !sigma || !out || n < 2) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        check_cfg(cfg);
        if (s->impl.ctx != &ctx->impl) throw Error{AUSAXS_ERR_ARGUMENT, "structure belongs to another context"};
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const ausaxs_debye_params b = default_params(base);
        FitArgs F = fit_search(*cfg, options, b);
        const size_t vec = align_up((size_t)n * 8, 256);
        C.io.ensure(9 * vec + 256);
        char* io = C.io.as<char>();
        double* prof = reinterpret_cast<double*>(io);
        double* Iu = reinterpret_cast<double*>(io + 6 * vec);
        F.Iw = reinterpret_cast<double*>(io + 7 * vec);
        F.W = reinterpret_cast<double*>(io + 8 * vec);
        F.out = reinterpret_cast<double*>(io + 9 * vec);
        s->impl.enqueue_histogram(*cfg);
        DebyeArgs A = s->impl.debye_args(*cfg, q, n, unit_params(b), Iu, prof);
        run_debye(C, A, cfg->manager == AUSAXS_MANAGER_FFGRID ? 7 : 1, s->impl.plan.tc, 1);
        F.nq = n;
        F.q = q;
        F.P = prof;
        F.y = I;
        F.sigma = sigma;
        F.I_fit = I_fit;
        fit_launch(F, C.stream);
        C.check_launch("fit");
        unsigned long long overflow = 0;
        AUSAXS_CUDA(cudaMemcpyAsync(&overflow, A.overflow, 8, cudaMemcpyDeviceToHost, C.stream));
        read_fit(C, F.out, out);
        if (overflow)
            throw Error{AUSAXS_ERR_BIN_OVERFLOW, "pair distances beyond bin_count * bin_width; increase settings::axes::bin_count"};
    });
}

// Excluded-volume dummies of the molecular grid (RawGridExv::create on the expanded grid) and the grid
// volume; the scratch structure takes the census, the context's grid workspace is reused.
int ausaxs_gpu_grid_exv(ausaxs_gpu_ctx* ctx, const float* atoms, int32_t n_atoms, const float* waters,
                        int32_t n_waters, int32_t host_pointers, float* exv_out, int64_t capacity, int64_t* n_exv,
                        double* volume) {
    return guarded([&] {
        if (!ctx || !n_exv || n_atoms < 0 || n_waters < 0 || (n_atoms && !atoms) || (n_waters && !waters) ||
            (capacity > 0 && !exv_out))
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        const bool host = host_pointers != 0;
        *n_exv = 0;
        if (volume) *volume = 0;
        Structure& S = scratch(C);  // census and validation of the points (form-factor types, finite coordinates)
        S.load(atoms, n_atoms, waters, n_waters, nullptr, 0, 1, host);
        GridExv& g = grid_workspace(C);
        // device output: the dummies go straight to exv_out; a short buffer fails once the count is known
        float4* direct = (!host && capacity > 0) ? reinterpret_cast<float4*>(exv_out) : nullptr;
        try {
            g.run(C, S.raw_a.as<float4>(), n_atoms, S.raw_w.as<float4>(), n_waters, S.lo, S.hi, capacity > 0, direct,
                  capacity);
        } catch (const Error&) {
            *n_exv = g.count;
            if (volume) *volume = g.volume;
            throw;
        }
        *n_exv = g.count;
        if (volume) *volume = g.volume;
        if (host && capacity > 0 && g.count > 0) {
            if (capacity < g.count) throw Error{AUSAXS_ERR_CAPACITY, "exv_out holds fewer records than the grid has dummies"};
            AUSAXS_CUDA(cudaMemcpyAsync(exv_out, g.points.p, (size_t)g.count * 16, cudaMemcpyDeviceToHost, C.stream));
        }
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    });
}


int ausaxs_hydrate_axes(const double* atoms, int64_t n_atoms, double* axes) {
    return guarded([&] {
        if (!axes || n_atoms < 0 || (n_atoms && !atoms)) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        double gmin[3];
        int bins[3];
        hydrate_axes(atoms, n_atoms, gmin, bins);
        for (int d = 0; d < 3; ++d) axes[d] = gmin[d], axes[3 + d] = bins[d];
    });
}


// Hydration shell (RadialHydration) on a fresh grid: the atoms, types and noise table go to the
// context's hydration workspace, the waters and their candidate indices come back.
int ausaxs_gpu_hydrate(ausaxs_gpu_ctx* ctx, const double* atoms, const int32_t* ff_types, int64_t n_atoms,
                       const double* axes, const double* noise, uint64_t noise_seed, double* waters_out,
                       int64_t capacity, int64_t* n_waters, int64_t* candidates_out, int32_t* rounds) {
    return guarded([&] {
        if (!ctx || bad_hydrate_args(atoms, ff_types, n_atoms, waters_out, capacity, n_waters))
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        *n_waters = 0;
        if (rounds) *rounds = 0;
        double gmin[3];
        int bins[3];
        if (axes) read_axes(axes, gmin, bins);
        else hydrate_axes(atoms, n_atoms, gmin, bins);
        check_hydration_atoms(atoms, ff_types, n_atoms, gmin, bins);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        Hydrator& H = hydrator(C);
        double *d_atoms, *d_noise;
        int32_t* d_ff;
        stage_hydration_inputs(C, H, atoms, ff_types, n_atoms, noise, &d_atoms, &d_ff, &d_noise);
        H.run(C, d_atoms, d_ff, n_atoms, gmin, bins, d_noise, noise ? 0ull : (unsigned long long)noise_seed);
        read_waters(C, H, waters_out, capacity, n_waters, candidates_out, rounds);
    });
}

// The same on device-resident atoms, types and noise, writing device buffers (no host staging).
int ausaxs_gpu_hydrate_device(ausaxs_gpu_ctx* ctx, const double* atoms, const int32_t* ff_types, int64_t n_atoms,
                              const double* axes, const double* noise, uint64_t noise_seed, double* waters_out,
                              int64_t capacity, int64_t* n_waters, int64_t* candidates_out, int32_t* rounds) {
    return guarded([&] {
        if (!ctx || !axes || bad_hydrate_args(atoms, ff_types, n_atoms, waters_out, capacity, n_waters))
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        *n_waters = 0;
        if (rounds) *rounds = 0;
        double gmin[3];
        int bins[3];
        read_axes(axes, gmin, bins);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        Hydrator& H = hydrator(C);
        H.run(C, atoms, ff_types, n_atoms, gmin, bins, noise, noise ? 0ull : (unsigned long long)noise_seed);
        *n_waters = H.count;
        if (rounds) *rounds = H.rounds;
        if (capacity > 0 && H.count > 0) {
            if (capacity < H.count) throw Error{AUSAXS_ERR_CAPACITY, "waters_out holds fewer waters than were placed"};
            AUSAXS_CUDA(cudaMemcpyAsync(waters_out, H.waters(), (size_t)H.count * 24, cudaMemcpyDeviceToDevice, C.stream));
            if (candidates_out)
                AUSAXS_CUDA(cudaMemcpyAsync(candidates_out, H.candidates(), (size_t)H.count * 8, cudaMemcpyDeviceToDevice,
                                            C.stream));
        }
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
    });
}

int ausaxs_gpu_ctx_hydration_stats(ausaxs_gpu_ctx* ctx, int64_t* survivors, int32_t* rounds) {
    return guarded([&] {
        if (!ctx) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        const Ctx& C = ctx->impl;
        if (survivors) *survivors = C.hyd ? C.hyd->survivors : 0;
        if (rounds) *rounds = C.hyd ? C.hyd->rounds : 0;
    });
}

int ausaxs_gpu_hydration_grid_create(ausaxs_gpu_ctx* ctx, const double* axes, ausaxs_gpu_hydration_grid** out) {
    return guarded([&] {
        if (!ctx || !axes || !out) throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        *out = nullptr;
        auto g = std::make_unique<ausaxs_gpu_hydration_grid>();
        g->ctx = ctx;
        read_axes(axes, g->gmin, g->bins);
        Ctx& C = ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        g->cell_bytes = align_up((size_t)g->bins[0] * g->bins[1] * g->bins[2], 256);
        g->cells.ensure(g->cell_bytes + 256);
        AUSAXS_CUDA(cudaMemsetAsync(g->cells.p, 0, g->cell_bytes + 8, C.stream));
        AUSAXS_CUDA(cudaStreamSynchronize(C.stream));
        *out = g.release();
    });
}

int ausaxs_gpu_hydration_grid_destroy(ausaxs_gpu_hydration_grid* g) {
    return guarded([&] {
        if (!g) return;
        AUSAXS_CUDA(cudaSetDevice(g->ctx->impl.device));
        AUSAXS_CUDA(cudaStreamSynchronize(g->ctx->impl.stream));
        delete g;
    });
}


int ausaxs_gpu_hydration_grid_add(ausaxs_gpu_hydration_grid* g, const double* atoms, const int32_t* ff_types,
                                  int64_t n_atoms) {
    return hydration_grid_edit(g, atoms, ff_types, n_atoms, true);
}

int ausaxs_gpu_hydration_grid_remove(ausaxs_gpu_hydration_grid* g, const double* atoms, const int32_t* ff_types,
                                     int64_t n_atoms) {
    return hydration_grid_edit(g, atoms, ff_types, n_atoms, false);
}

int ausaxs_gpu_hydration_grid_hydrate(ausaxs_gpu_hydration_grid* g, const double* atoms, const int32_t* ff_types,
                                      int64_t n_atoms, const double* noise, uint64_t noise_seed, double* waters_out,
                                      int64_t capacity, int64_t* n_waters, int64_t* candidates_out, int32_t* rounds) {
    return guarded([&] {
        if (!g || bad_hydrate_args(atoms, ff_types, n_atoms, waters_out, capacity, n_waters))
            throw Error{AUSAXS_ERR_ARGUMENT, "invalid argument"};
        *n_waters = 0;
        if (rounds) *rounds = 0;
        check_hydration_atoms(atoms, ff_types, n_atoms, g->gmin, g->bins);
        Ctx& C = g->ctx->impl;
        AUSAXS_CUDA(cudaSetDevice(C.device));
        Hydrator& H = hydrator(C);
        double *d_atoms, *d_noise;
        int32_t* d_ff;
        stage_hydration_inputs(C, H, atoms, ff_types, n_atoms, noise, &d_atoms, &d_ff, &d_noise);
        H.generate(C, g->cells.as<uint8_t>(), g->gmin, g->bins, d_atoms, d_ff, n_atoms, d_noise,
                   noise ? 0ull : (unsigned long long)noise_seed);
        read_waters(C, H, waters_out, capacity, n_waters, candidates_out, rounds);
    });
}

}  // extern "C"
