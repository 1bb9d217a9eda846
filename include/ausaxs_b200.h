/*
 * ausaxs_b200 -- C ABI of the B200 (sm_100a) Debye hot path.
 *
 * The two stages of AUSAXS's hot path sit behind these entry points:
 *
 *   1. pair-distance histograms, i.e. what
 *        hist::IHistogramManager::calculate_all()
 *      returns (include/core/hist/histogram_manager/IHistogramManager.h:16-29) for the
 *      managers HistogramManagerMT, HistogramManagerMTFFAvg, HistogramManagerMTFFExplicit and
 *      HistogramManagerMTFFGrid (one .cpp per manager in source/core/hist/histogram_manager/);
 *   2. the Debye transform, i.e.
 *        ICompositeDistanceHistogram::debye_transform() and get_profile_*()
 *      (include/core/hist/intensity_calculator/ICompositeDistanceHistogram.h:24-71,
 *       ICompositeDistanceHistogramExv.h:12-107), evaluated at caller-given q.
 *
 * Conventions (all entry points):
 *   - every function returns an int status: AUSAXS_OK (0) or one of the AUSAXS_ERR_* codes; the
 *     message of the last failure on the calling thread is returned by ausaxs_gpu_last_error().
 *     This mirrors the reference's C API, where exceptions become a non-zero *status plus a
 *     last-error string (include/api/api/api_helper.h:15-45).  No exception crosses this ABI.
 *   - point arrays are the reference's compact 16-byte records, n x {float x, y, z; w | ff}
 *     (include/core/hist/detail/data/CompactCoordinatesXYZW.h:131-134 for weights,
 *     CompactCoordinatesXYZFF.h for the int32 form-factor type, form_factor_t numbering
 *     include/core/form_factor/FormFactorType.h:14-37).  A caller holding
 *     hist::detail::CompactCoordinates can pass get_data().data() directly.
 *   - ausaxs_gpu_histogram / _debye / _profile take host pointers and copy inside; the
 *     ausaxs_gpu_structure_* entry points work on device-resident structures.
 *   - output buffers are always caller-allocated.
 *   - a context is not thread-safe; use one context per host thread.
 */
#ifndef AUSAXS_B200_H
#define AUSAXS_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define AUSAXS_API __attribute__((visibility("default")))
#else
#define AUSAXS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    AUSAXS_OK = 0,
    AUSAXS_ERR_ARGUMENT = 1,     /* invalid argument (null pointer, negative size, ...)           */
    AUSAXS_ERR_CUDA = 2,         /* a CUDA runtime call failed                                     */
    AUSAXS_ERR_BIN_OVERFLOW = 3, /* a pair distance fell outside bin_count bins (the reference's   */
                                 /* HistogramSettings.cpp:51-61 only warns; here it is an error)    */
    AUSAXS_ERR_FORM_FACTOR = 4,  /* a form-factor type outside [0, 15) (CompactCoordinatesFF.h:24) */
    AUSAXS_ERR_CAPACITY = 5,     /* request exceeds a capacity (memory budget, slots, ...)          */
    AUSAXS_ERR_TIMEOUT = 6,      /* a bounded wait ran out                                          */
    AUSAXS_ERR_NOT_FOUND = 7     /* unknown handle / request id                                     */
};

/* settings::hist::HistogramManagerChoice (include/core/settings/HistogramSettings.h) */
enum {
    AUSAXS_MANAGER_MT = 1,         /* HistogramManagerMT: weights, Simple excluded volume       */
    AUSAXS_MANAGER_FFAVG = 2,      /* HistogramManagerMTFFAvg: form factors, average exv         */
    AUSAXS_MANAGER_FFEXPLICIT = 3, /* HistogramManagerMTFFExplicit: form factors, no exv rows    */
    AUSAXS_MANAGER_FFGRID = 4      /* HistogramManagerMTFFGrid: form factors, grid exv dummies   */
};

typedef struct ausaxs_gpu_ctx ausaxs_gpu_ctx;

/* Create a context on a CUDA device (its own stream and device workspace). */
AUSAXS_API int ausaxs_gpu_ctx_create(int device, ausaxs_gpu_ctx** out);
AUSAXS_API int ausaxs_gpu_ctx_destroy(ausaxs_gpu_ctx* ctx);
/* Use an existing CUDA stream (cudaStream_t passed as void*) for all later work; NULL = own stream. */
AUSAXS_API int ausaxs_gpu_ctx_set_stream(ausaxs_gpu_ctx* ctx, void* stream);
/* Number of kernels this context has launched (instrumentation for benchmarks). */
AUSAXS_API int64_t ausaxs_gpu_ctx_launch_count(const ausaxs_gpu_ctx* ctx);
AUSAXS_API const char* ausaxs_gpu_last_error(void);
/*
 * Optional kernel timing (instrumentation, no counterpart in the reference): with timing enabled,
 * every later launch of a kernel class is bracketed by CUDA events on the context's stream.
 * ausaxs_gpu_ctx_kernel_time synchronises the stream and returns the accumulated device time (ms)
 * and number of launches of one class: 0 = pair histograms, 1 = finalisation, 2 = FP64 Debye
 * epilogue, 3 = tensor-core Debye contraction, 4 = grid excluded-volume kernels, 5 = hydration kernels.
 * ausaxs_gpu_ctx_fp64_columns: how many q values the last ausaxs_gpu_debye call evaluated in FP64
 * (all of them with precision 1; those whose tensor-core error estimate exceeded the tolerance with
 * precision 0).
 */
AUSAXS_API int ausaxs_gpu_ctx_enable_timing(ausaxs_gpu_ctx* ctx, int32_t enable);
AUSAXS_API int ausaxs_gpu_ctx_kernel_time(ausaxs_gpu_ctx* ctx, int32_t kernel_class, double* ms, int64_t* launches);
AUSAXS_API int ausaxs_gpu_ctx_fp64_columns(ausaxs_gpu_ctx* ctx, int32_t* n);
/* Per q of the last ausaxs_gpu_debye call with precision 0: the rigorous bound on the relative error
 * of the tensor-core I(q) (before any FP64 re-evaluation); INFINITY where none was formed. */
AUSAXS_API int ausaxs_gpu_ctx_tc_error_estimate(ausaxs_gpu_ctx* ctx, double* out, int32_t nq);

/*
 * Histogram configuration: the global settings the reference reads during calculate_all().
 *   bin_width, bin_count : settings::axes::bin_width / bin_count (HistogramSettings.cpp:38-80);
 *                          the pair bin is round(float(d) * float(1/bin_width))
 *                          (include/core/hist/detail/data/WidthControllers.h:10-26)
 *   weighted_bins        : settings::hist::weighted_bins (mean distance per bin as d-axis)
 *   z_exv                : FFAvg only, V_grid * rho_w / N_atoms (HistogramManagerMTFFAvg.cpp:351-364)
 */
typedef struct {
    int32_t manager;
    int32_t weighted_bins;
    double bin_width;
    int32_t bin_count;
    double z_exv;
} ausaxs_hist_config;

/*
 * Histogram result, in the reference's layouts, truncated to max_bin bins
 * (HistogramManagerMT.cpp:47-58): every row below is written with stride max_bin.
 * All pointers are caller-allocated host buffers with room for bin_count bins per row.
 *   MT    : aa, aw, ww, tot = weighted counts (get_aa_counts/get_aw_counts/get_ww_counts/get_counts)
 *   FF*   : aa = [15][15] rows (get_raw_aa_counts_by_ff), aw = [15] rows (get_raw_aw_counts_by_ff),
 *           ww (get_raw_ww_counts_by_ff), tot = p_tot counts
 *   d_axis: DistanceHistogram::get_d_axis() (weighted bin centres, bin 0 pinned to 0)
 *   FFGRID: d_axis_ax / d_axis_xx = CompositeDistanceHistogramFFGrid::get_d_axis_ax/_xx
 */
typedef struct {
    int32_t max_bin;
    int64_t pairs;          /* pair evaluations performed                         */
    int64_t overflow_pairs; /* pairs whose bin fell outside bin_count (then ERR 3) */
    double* aa;
    double* aw;
    double* ww;
    double* tot;
    double* d_axis;
    double* d_axis_ax;
    double* d_axis_xx;
} ausaxs_hist_result;

/* n_exv value asking ausaxs_gpu_histogram / ausaxs_gpu_profile (FFGRID) to take the excluded-volume
 * dummies from the structure's molecular grid, as the reference does (see ausaxs_gpu_grid_exv). */
#define AUSAXS_EXV_FROM_GRID (-1)

/*
 * IHistogramManager::calculate_all() for one structure (host buffers).
 * atoms: n_atoms records, waters: n_waters records, exv: n_exv excluded-volume dummies (FFGRID only;
 * RawGridExv::create supplies these in the reference, source/core/grid/exv/RawGridExv.cpp:10-59).
 * FF managers read the int32 form-factor type from the 4th word, MT reads the float weight.
 * FFGRID with n_exv = AUSAXS_EXV_FROM_GRID generates the dummies on the device (ausaxs_gpu_grid_exv);
 * FFAVG with cfg->z_exv < 0 takes Z_exv = V_grid * rho_w / N_atoms from the grid volume, as
 * HistogramManagerMTFFAvg does with Molecule::get_volume_grid().
 */
AUSAXS_API int ausaxs_gpu_histogram(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const float* atoms, int32_t n_atoms,
                         const float* waters, int32_t n_waters, const float* exv, int32_t n_exv,
                         ausaxs_hist_result* out);

/*
 * Free parameters of the composite histograms
 * (CompositeDistanceHistogramFFAvgBase.cpp:216-238: cw = water scaling, cx = excluded-volume
 * scaling, crho = solvent density scaling, Debye-Waller sigmas for atoms and exv).
 * grid_width: settings::grid::exv::width, the FFGRID dummy volume is grid_width^3.
 * precision: 0 = split-BF16 tensor-core contraction with FP64 recomputation of every q whose
 *            estimated error exceeds tolerance; 1 = FP64 on CUDA cores for every q; 3 = exact-
 *            accumulation tensor-core contraction (int8 digits of the histogram rows and of Taylor
 *            tables of sinc shared by every call on the same q grid, s32 sums) with a rigorous bound
 *            per q and FP64 recomputation of every q whose bound exceeds tolerance; 2 = automatic:
 *            3 when the transform has at least 8e6 row x bin x q products (below that the
 *            contraction's fixed cost exceeds the FP64 transform's), else 1.
 */
typedef struct {
    double cw, cx, crho, dw_atomic, dw_exv;
    double grid_width;
    int32_t precision;
    double tolerance; /* relative I(q) error target for precision 0, 2, 3 (default 1e-5 when <= 0) */
} ausaxs_debye_params;

/*
 * debye_transform() of a histogram previously returned by ausaxs_gpu_histogram (host buffers),
 * evaluated at the caller's q values (the generalised-q form of
 * CompositeDistanceHistogramFFAvgBase::debye_transform, :57-76).
 * Iq: n_q values; profiles (optional, 6 x n_q): {aa, ax, aw, xx, wx, ww} as get_profile_*().
 */
AUSAXS_API int ausaxs_gpu_debye(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const ausaxs_hist_result* hist,
                     const double* q, int32_t n_q, const ausaxs_debye_params* params, double* Iq, double* profiles);

/*
 * Coordinates -> I(q) in one call (Molecule::get_histogram()->debye_transform(), host buffers):
 * histogram and transform stay on the device; only I(q) (and optional profiles) come back.
 */
AUSAXS_API int ausaxs_gpu_profile(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const float* atoms, int32_t n_atoms,
                       const float* waters, int32_t n_waters, const float* exv, int32_t n_exv, const double* q,
                       int32_t n_q, const ausaxs_debye_params* params, double* Iq, double* profiles);

/*
 * Device-resident structures.  A structure keeps its points in device memory; its first profile
 * under a configuration builds a launch plan (allocation, one synchronisation), every later
 * profile is a fixed sequence of kernels on the context's stream with no allocation, copy or
 * synchronisation (so it can be captured in a CUDA graph).  This is the analogue of the
 * reference's Molecule owning its histogram manager (source/core/data/Molecule.cpp:67-75, 236).
 *
 * ausaxs_gpu_structure_create: points as in ausaxs_gpu_histogram; host_pointers != 0 means the
 *   arrays are host memory, otherwise device memory of the context's device.  ff_typed != 0: the
 *   4th word is the int32 form-factor type (FF managers), else the float weight (MT).  One
 *   synchronisation (point census: bounding box, type counts, validation).  With ff_typed and
 *   n_exv = AUSAXS_EXV_FROM_GRID the structure's dummies are those of its molecular grid, generated
 *   on the device once (the reference's Molecule caches its grid the same way, Molecule.cpp:246-248);
 *   three synchronisations.
 * ausaxs_gpu_structure_profile: q, Iq and profiles are device pointers.  A histogram that lost
 *   pairs to bin overflow yields NaN in Iq.
 * ausaxs_gpu_structure_histogram: host result as ausaxs_gpu_histogram (synchronises).
 */
typedef struct ausaxs_gpu_structure ausaxs_gpu_structure;

AUSAXS_API int ausaxs_gpu_structure_create(ausaxs_gpu_ctx* ctx, int32_t ff_typed, const float* atoms, int32_t n_atoms,
                                const float* waters, int32_t n_waters, const float* exv, int32_t n_exv,
                                int32_t host_pointers, ausaxs_gpu_structure** out);
AUSAXS_API int ausaxs_gpu_structure_destroy(ausaxs_gpu_structure* s);
AUSAXS_API int ausaxs_gpu_structure_profile(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                                 const double* q, int32_t n_q, const ausaxs_debye_params* params, double* Iq,
                                 double* profiles);
AUSAXS_API int ausaxs_gpu_structure_histogram(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                                   ausaxs_hist_result* out);

/*
 * Batched profiles of many independent structures (FFAVG or FFGRID).  The reference computes one
 * structure per HistogramManagerMTFFAvg::calculate_all() (HistogramManagerMTFFAvg.cpp:194-372) and
 * debye_transform(); a batch gives every structure's I(q) from one replay of a captured CUDA graph:
 * the pair jobs of all structures in shared persistent launches, one batched finalisation, one
 * batched FP64 transform.
 *
 * ausaxs_gpu_batch_create: points of structure i are rows [off[i], off[i+1]) of the concatenated
 *   {x, y, z, ff} arrays (offsets have n_structures + 1 entries; exv/exv_offsets only for FFGRID);
 *   z_exv[i] (may be null: cfg->z_exv for all) is the FFAVG excluded-volume charge per atom.  One
 *   synchronisation per structure (census) at creation.
 * ausaxs_gpu_batch_autotune: times every pair-plan candidate on this batch, keeps the fastest and
 *   remembers it for batches of the same shape; choice and per-candidate milliseconds are returned
 *   (times_ms may be null).  ausaxs_gpu_batch_candidate describes a candidate.
 * ausaxs_gpu_batch_profile_device: q and Iq[n_structures * n_q] are device pointers; enqueues one
 *   graph launch on the context's stream (the graph is captured on the first call and again when
 *   q, Iq, n_q or the parameters change).  params->precision 1: FP64 transform for every q; 0, 2, 3:
 *   the exact-accumulation tensor-core transform (int8 digit products of the histogram rows and of
 *   shared Taylor tables of sinc, s32 sums) with a rigorous error bound per q, and the FP64
 *   transform for every q whose bound exceeds params->tolerance times |I(q)|.  Any bin overflow in
 *   the batch makes every Iq NaN.
 * ausaxs_gpu_batch_profile: host q and Iq (synchronises; bin overflow is an error).
 * ausaxs_gpu_batch_pair_time: device milliseconds of the pair stage (accumulator clearing and every
 *   pair launch) of the last profile, from events recorded inside the captured graph (waits for it).
 * ausaxs_gpu_batch_histogram: structure `index`'s histograms from the last profile, as
 *   ausaxs_gpu_structure_histogram.
 * ausaxs_gpu_batch_fp64_columns: (structure, q) values of the last profile that the FP64 transform
 *   recomputed because their tensor-core error bound exceeded the tolerance (waits for the profile).
 * ausaxs_gpu_batch_set_points (FFAVG batches): new x, y, z for every atom and water, in the creation
 *   layout (same offsets, so the same arrays' shapes); each atom's form-factor type must be the one it
 *   was created with; z_exv (host, n_structures values, may be null: kept) replaces the FFAVG
 *   excluded-volume charges.  Plans, job tables and the captured graph are kept, so the next profile is one
 *   graph replay.  Bins stay those planned from the creation coordinates: a pair that now lies beyond
 *   them is a bin overflow (error from ausaxs_gpu_batch_profile, NaN from _profile_device; create the
 *   batch again).  A point whose type changed or that has a non-finite coordinate is left as it was
 *   and counted: host_pointers = 1 synchronises and fails with AUSAXS_ERR_ARGUMENT, and every later
 *   profile fails (or is NaN) until a set_points call without rejections.  host_pointers = 0 reads
 *   device arrays and does not synchronise.
 */
typedef struct ausaxs_gpu_batch ausaxs_gpu_batch;

AUSAXS_API int ausaxs_gpu_batch_create(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, int32_t n_structures,
                                       const float* atoms, const int64_t* atom_offsets, const float* waters,
                                       const int64_t* water_offsets, const float* exv, const int64_t* exv_offsets,
                                       const double* z_exv, int32_t host_pointers, ausaxs_gpu_batch** out);
AUSAXS_API int ausaxs_gpu_batch_destroy(ausaxs_gpu_batch* b);
AUSAXS_API int ausaxs_gpu_batch_autotune(ausaxs_gpu_batch* b, int32_t* choice, double* times_ms, int32_t n_times);
AUSAXS_API int ausaxs_gpu_batch_candidate(int32_t index, int32_t* tile_small, int32_t* tile_large, int32_t* threshold,
                                          int32_t* by_class);
AUSAXS_API int ausaxs_gpu_batch_profile_device(ausaxs_gpu_batch* b, const double* q, int32_t n_q,
                                               const ausaxs_debye_params* params, double* Iq);
AUSAXS_API int ausaxs_gpu_batch_profile(ausaxs_gpu_batch* b, const double* q, int32_t n_q,
                                        const ausaxs_debye_params* params, double* Iq);
AUSAXS_API int ausaxs_gpu_batch_pair_time(ausaxs_gpu_batch* b, double* ms);
AUSAXS_API int ausaxs_gpu_batch_histogram(ausaxs_gpu_batch* b, int32_t index, ausaxs_hist_result* out);
AUSAXS_API int ausaxs_gpu_batch_fp64_columns(ausaxs_gpu_batch* b, int64_t* n);
AUSAXS_API int ausaxs_gpu_batch_set_points(ausaxs_gpu_batch* b, const float* atoms, const float* waters,
                                           const double* z_exv, int32_t host_pointers);

/*
 * Fit of one free parameter of a composite histogram to measured data: fitter::SmartFitter::fit()
 * (source/core/fitter/SmartFitter.cpp:147-176) with the minimiser of a build without dlib, the
 * golden-section search mini::Golden (source/core/mini/Golden.cpp:26-74).  Every trial value is scored
 * by the linear fit I ~ a I_model + b with weights 1/sigma^2 and its chi2
 * (fitter::detail::LinearLeastSquares, LinearLeastSquares.cpp:26-78); the model is evaluated at the
 * data's own q values (the reference splines its fixed q axis onto them, which is the identity when
 * the data lie on that axis).  One FP64 transform gives the six unit profiles, the whole search then
 * runs in one kernel.
 *
 * parameter: 0 water scaling cw, 1 excluded-volume scaling cx, 2 solvent density crho, 3 atomic and
 *   4 excluded-volume Debye-Waller sigma (SmartFitter's enabled parameter; the others keep their
 *   values from `base`, whose precision and tolerance fields are not used).  lo == hi selects the
 *   reference's limits for the parameter (cw [0, 10], cx [0.92, 1.08], crho [0.5, 2], Debye-Waller
 *   [0, 5]); tolerance <= 0 selects 1e-4 (mini::Minimizer::tol).  The Simple (MT) histogram has cw
 *   only.
 * evaluations counts the trials as the reference reports them (the final evaluation at value
 * excluded).  I_fit (optional, n values) receives a I_model + b at the fitted value.
 */
typedef struct {
    int32_t parameter;
    double lo, hi;
    double tolerance;
} ausaxs_fit_options;

typedef struct {
    double value;        /* the fitted parameter: centre of the final interval */
    double a, b;         /* I ~ a I_model + b at value */
    double a_err, b_err; /* sqrt of the diagonal of the normal equations' inverse */
    double chi2;
    int32_t evaluations;
} ausaxs_fit_result;

/* A histogram previously returned by ausaxs_gpu_histogram (host buffers); q, I, sigma: host, n values. */
AUSAXS_API int ausaxs_gpu_fit(ausaxs_gpu_ctx* ctx, const ausaxs_hist_config* cfg, const ausaxs_hist_result* hist,
                              const double* q, const double* I, const double* sigma, int32_t n,
                              const ausaxs_debye_params* base, const ausaxs_fit_options* options,
                              ausaxs_fit_result* out, double* I_fit);
/* A device-resident structure (its histogram is computed on the device); q, I, sigma and I_fit are
 * device arrays; out is host memory (synchronises). */
AUSAXS_API int ausaxs_gpu_structure_fit(ausaxs_gpu_ctx* ctx, ausaxs_gpu_structure* s, const ausaxs_hist_config* cfg,
                                        const double* q, const double* I, const double* sigma, int32_t n,
                                        const ausaxs_debye_params* base, const ausaxs_fit_options* options,
                                        ausaxs_fit_result* out, double* I_fit);

/*
 * hist::distance_calculator::SimpleCalculator<weighted_bins = true> (include/core/hist/
 * distance_calculator/SimpleCalculator.h:37-92) on the device: the distance calculator that
 * HistogramManagerMT, SymmetryManagerMT and PartialSymmetryManagerMT issue their work to.
 *   enqueue_self(points, n, scaling, merge_id): the pairs i < j of one weighted point set
 *     ({x, y, z, w} records, host memory), each with factor 2 * scaling, plus the diagonal
 *     scaling * sum(w*w) in bin 0;
 *   enqueue_cross(points_1, n_1, points_2, n_2, scaling, merge_id): every pair of the two sets, factor
 *     2 * scaling (points_2 outer, points_1 inner, as the reference loops);
 *   merge_id: jobs with the same id accumulate into one result (self and cross ids are separate);
 *     -1 makes a result of its own whose id is its index; *result_index is the reference's return
 *     value (the result's position among those of its kind).
 * The arrays must stay valid and unchanged until run(), as in the reference; a set passed several
 * times (same pointer and size) is copied once.  run() executes every job in shared persistent
 * launches (synchronises) and clears the jobs; the results of the last run stay available:
 *   result_ids lists the merge ids of one kind (ascending);
 *   result(cross, merge_id, ...) gives, for each of the bin_count bins, the WeightedDistribution1D
 *     entry: value (weighted count), count and the sum of the pair distances (bin-centre sum).
 */
typedef struct ausaxs_gpu_calculator ausaxs_gpu_calculator;

AUSAXS_API int ausaxs_gpu_calculator_create(ausaxs_gpu_ctx* ctx, double bin_width, int32_t bin_count,
                                            ausaxs_gpu_calculator** out);
AUSAXS_API int ausaxs_gpu_calculator_destroy(ausaxs_gpu_calculator* c);
AUSAXS_API int ausaxs_gpu_calculator_enqueue_self(ausaxs_gpu_calculator* c, const float* points, int32_t n,
                                                  int32_t scaling, int32_t merge_id, int32_t* result_index);
AUSAXS_API int ausaxs_gpu_calculator_enqueue_cross(ausaxs_gpu_calculator* c, const float* points_1, int32_t n_1,
                                                   const float* points_2, int32_t n_2, int32_t scaling,
                                                   int32_t merge_id, int32_t* result_index);
AUSAXS_API int ausaxs_gpu_calculator_run(ausaxs_gpu_calculator* c, int32_t* n_self, int32_t* n_cross);
AUSAXS_API int ausaxs_gpu_calculator_result_ids(ausaxs_gpu_calculator* c, int32_t cross, int32_t* ids,
                                                int32_t capacity, int32_t* n);
AUSAXS_API int ausaxs_gpu_calculator_result(ausaxs_gpu_calculator* c, int32_t cross, int32_t merge_id, double* value,
                                            double* count, double* distance_sum);

/*
 * Excluded-volume dummies of a structure's molecular grid: grid::exv::RawGridExv::create
 * (source/core/grid/exv/RawGridExv.cpp:10-59) on the expanded grid that
 * HistogramManagerMTFFGrid::calculate_all() uses, with the reference's default grid settings (1 A
 * cells, rvol 2.15 A, exv width 1 A, AtomicOnly expansion; Grid.cpp:34-102, SphericalExpander.h:27-76),
 * and the grid volume Molecule::get_volume_grid() returns (A^3).  atoms {x,y,z,ff} and waters
 * {x,y,z,w} are records in host memory (host_pointers != 0) or in device memory of the context's
 * device, as is exv_out.  Dummies are written as {x, y, z, 0} records in the reference's order
 * (x-major sweep) when capacity > 0; *n_exv is their count, set also when the call fails with
 * AUSAXS_ERR_CAPACITY because capacity is too small.  Synchronises the context's stream.
 */
AUSAXS_API int ausaxs_gpu_grid_exv(ausaxs_gpu_ctx* ctx, const float* atoms, int32_t n_atoms, const float* waters,
                                   int32_t n_waters, int32_t host_pointers, float* exv_out, int64_t capacity,
                                   int64_t* n_exv, double* volume);

/*
 * Hydration shell: the waters data::Molecule::generate_new_hydration() places with the reference's
 * default strategy, hydrate::RadialHydration without culling
 * (source/core/hydrate/generation/RadialHydration.cpp:43-206, GridBasedHydration.cpp:34-79), as
 * the rigid-body loop calls it after every move (source/rigidbody/controller/SimpleController.cpp:76).
 *   atoms: n_atoms x {x, y, z} (double, host memory) in the order the generator visits them (the
 *     grid's member order: bodies in order, a body that was moved appended after the others);
 *     ff_types: their form-factor types (1-14 or 16, FormFactorType.h:14-33).
 *   axes: {min x, y, z, bins x, y, z} of the grid (1 A cells), or null for the axes Grid(bodies)
 *     builds around these atoms (ausaxs_hydrate_axes); every atom must lie inside.
 *   noise: n_atoms x 26 x 3 displacements, one row per candidate in candidate order (the reference
 *     draws one from its noise generator per candidate), or null: then noise_seed != 0 draws
 *     Gaussian displacements of sigma 0.75 A on the device (a stream of its own, not the
 *     reference's), and noise_seed == 0 means none.
 *   Writes the waters (x, y, z, double) in the reference's order into waters_out and, when not null,
 *   their candidate indices (atom * 26 + direction, so the waters of each body can be told apart)
 *   into candidates_out, when capacity suffices; *n_waters is their count, set also when the call
 *   fails with AUSAXS_ERR_CAPACITY.  *rounds (may be null): the resolution rounds the device took.
 *   Synchronises the context's stream.
 */
#define AUSAXS_HYDRATE_DIRECTIONS 26
AUSAXS_API int ausaxs_gpu_hydrate(ausaxs_gpu_ctx* ctx, const double* atoms, const int32_t* ff_types, int64_t n_atoms,
                                  const double* axes, const double* noise, uint64_t noise_seed, double* waters_out,
                                  int64_t capacity, int64_t* n_waters, int64_t* candidates_out, int32_t* rounds);
/* ausaxs_gpu_hydrate on device memory of the context's device: atoms, ff_types, noise, waters_out and
 * candidates_out are device pointers; axes (host, 6 doubles) must be given.  The form-factor types are
 * not checked (a type without a radius counts as radius 0); an atom outside the axes fails the call. */
AUSAXS_API int ausaxs_gpu_hydrate_device(ausaxs_gpu_ctx* ctx, const double* atoms, const int32_t* ff_types,
                                         int64_t n_atoms, const double* axes, const double* noise, uint64_t noise_seed,
                                         double* waters_out, int64_t capacity, int64_t* n_waters,
                                         int64_t* candidates_out, int32_t* rounds);
/* Of the context's last hydration: the candidates that passed the static tests (their cell inside the
 * grid and not an atom's) and the resolution rounds. */
AUSAXS_API int ausaxs_gpu_ctx_hydration_stats(ausaxs_gpu_ctx* ctx, int64_t* survivors, int32_t* rounds);
/* The axes Grid(bodies) builds around n_atoms atoms (x, y, z doubles) for the hydration: {min x, y, z,
 * bins x, y, z} (Grid.cpp:34-102).  Host only. */
AUSAXS_API int ausaxs_hydrate_axes(const double* atoms, int64_t n_atoms, double* axes);

/*
 * A hydration grid kept across calls, as the reference keeps a molecule's grid::Grid between
 * rigid-body steps: create it with the axes, add every body's atoms (Grid::add with the volume
 * expansion), and per step remove the moved body at its old coordinates (Grid::remove: its atoms'
 * spheres of max(r_vdw, 2.15 A) lose their A_AREA / VOLUME marks, whatever other atoms cover them, and
 * its centre cells their A_CENTER mark; SingleTransform.cpp:20-69), add it at the new ones, and
 * hydrate.  hydrate takes the grid's member atoms in the grid's order (a re-added body comes last)
 * and otherwise behaves as ausaxs_gpu_hydrate.  Atoms must lie inside the axes.  The grid belongs to
 * the context it was made with (destroy the grid before the context); calls on it synchronise that
 * context's stream.
 */
typedef struct ausaxs_gpu_hydration_grid ausaxs_gpu_hydration_grid;
AUSAXS_API int ausaxs_gpu_hydration_grid_create(ausaxs_gpu_ctx* ctx, const double* axes, ausaxs_gpu_hydration_grid** out);
AUSAXS_API int ausaxs_gpu_hydration_grid_destroy(ausaxs_gpu_hydration_grid* grid);
AUSAXS_API int ausaxs_gpu_hydration_grid_add(ausaxs_gpu_hydration_grid* grid, const double* atoms,
                                             const int32_t* ff_types, int64_t n_atoms);
AUSAXS_API int ausaxs_gpu_hydration_grid_remove(ausaxs_gpu_hydration_grid* grid, const double* atoms,
                                                const int32_t* ff_types, int64_t n_atoms);
AUSAXS_API int ausaxs_gpu_hydration_grid_hydrate(ausaxs_gpu_hydration_grid* grid, const double* atoms,
                                                 const int32_t* ff_types, int64_t n_atoms, const double* noise,
                                                 uint64_t noise_seed, double* waters_out, int64_t capacity,
                                                 int64_t* n_waters, int64_t* candidates_out, int32_t* rounds);

/*
 * Rigid-body serving.  The reference's incremental manager, PartialHistogramManagerMT
 * (PartialHistogramManagerMT.cpp:42-170, 308-341), keeps per-body self partials and per-body-pair
 * cross partials and rebuilds the master from them after a body moves (Simple model only).  A server
 * keeps multi-body FFAVG assemblies on the device with the same decomposition; a request moves one
 * body (x <- R x + t, Body::rotate then Body::translate, source/core/data/Body.cpp:135-156, applied to
 * the body's current pose), recomputes the partials between that body and the others, and returns
 * I(q) plus the linear fit {a, b, sigma_a, sigma_b, chi2} against the assembly's target profile
 * (ausaxs_gpu_linear_lsq).  Each pair is evaluated with the full assembly's loop geometry, so the
 * histograms equal a full HistogramManagerMTFFAvg::calculate_all() of the moved assembly exactly.
 *
 * ausaxs_gpu_server_create: hbm_budget_bytes bounds the summed footprint of admitted assemblies;
 *   max_inflight bounds requests in flight; slots_per_assembly bounds one assembly's.
 * ausaxs_gpu_server_admit: bodies are rows [off[k], off[k+1]) of the concatenated host arrays
 *   (atoms {x,y,z,ff}, waters {x,y,z,w}; offsets have n_bodies + 1 entries); cfg->manager must be
 *   AUSAXS_MANAGER_FFAVG (cfg->z_exv as ausaxs_gpu_histogram); margin (A) widens the distance range
 *   beyond the initial bounding-box diagonal for later moves; q, params: the transform of every
 *   response; target/target_err (may be null: no fit, zeros) the fitted profile.  AUSAXS_ERR_CAPACITY
 *   when the footprint does not fit the free budget (footprint is returned either way).
 * ausaxs_gpu_server_submit: body -1 recomputes the current state without a move.  R is row-major
 *   3x3.  Returns a ticket, or AUSAXS_ERR_CAPACITY when no slot is free (retry after a completion).
 * ausaxs_gpu_server_poll / _wait: copy I(q) [n_q] and fit5 [5] (either may be null) when done; wait
 *   gives AUSAXS_ERR_TIMEOUT after timeout_ms.  A request whose pairs fell outside the distance range
 *   yields NaN in I(q), and so do all later requests of that assembly.
 * ausaxs_gpu_server_completed: up to `capacity` tickets whose results are ready (not consumed:
 *   collect them with poll).
 * ausaxs_gpu_server_body_center: the body's current centroid (for moves about it).
 * ausaxs_gpu_server_coordinates / _histogram: current coordinates (atoms with dense type indices
 *   in w) and histograms (as ausaxs_gpu_structure_histogram) after the assembly's last request.
 * One server per host thread.
 */
typedef struct ausaxs_gpu_server ausaxs_gpu_server;

AUSAXS_API int ausaxs_gpu_server_create(int32_t device, int64_t hbm_budget_bytes, int32_t max_inflight,
                                        int32_t slots_per_assembly, ausaxs_gpu_server** out);
AUSAXS_API int ausaxs_gpu_server_destroy(ausaxs_gpu_server* s);
/* Scheduling of requests: k in [1, 16] (default 2) requests in submission order, round robin over k
 * server streams, so at most k moves share the device (1: each move has it alone); 0 every assembly's
 * requests on its own two streams, so moves of all assemblies overlap on the device, moves of at most
 * the median size at high stream priority.  An assembly's requests stay in order. */
AUSAXS_API int ausaxs_gpu_server_set_policy(ausaxs_gpu_server* s, int32_t policy);
AUSAXS_API int ausaxs_gpu_server_admit(ausaxs_gpu_server* s, const ausaxs_hist_config* cfg, int32_t n_bodies,
                                       const float* atoms, const int64_t* atom_offsets, const float* waters,
                                       const int64_t* water_offsets, double margin, const double* q, int32_t n_q,
                                       const ausaxs_debye_params* params, const double* target,
                                       const double* target_err, int32_t* id, int64_t* footprint);
AUSAXS_API int ausaxs_gpu_server_release(ausaxs_gpu_server* s, int32_t id);
AUSAXS_API int ausaxs_gpu_server_usage(ausaxs_gpu_server* s, int64_t* used, int64_t* budget, int32_t* inflight);
AUSAXS_API int ausaxs_gpu_server_submit(ausaxs_gpu_server* s, int32_t id, int32_t body, const double* R,
                                        const double* t, int64_t* ticket);
AUSAXS_API int ausaxs_gpu_server_poll(ausaxs_gpu_server* s, int64_t ticket, int32_t* done, double* Iq, double* fit5);
AUSAXS_API int ausaxs_gpu_server_wait(ausaxs_gpu_server* s, int64_t ticket, int32_t timeout_ms, double* Iq,
                                      double* fit5);
/* Kernels launched for the admitted assemblies so far (instrumentation, as ausaxs_gpu_ctx_launch_count). */
AUSAXS_API int ausaxs_gpu_server_launch_count(ausaxs_gpu_server* s, int64_t* launches);
AUSAXS_API int ausaxs_gpu_server_completed(ausaxs_gpu_server* s, int64_t* tickets, int32_t capacity, int32_t* n);
AUSAXS_API int ausaxs_gpu_server_body_center(ausaxs_gpu_server* s, int32_t id, int32_t body, double* center);
AUSAXS_API int ausaxs_gpu_server_coordinates(ausaxs_gpu_server* s, int32_t id, float* atoms_xyzw, float* waters_xyzw);
AUSAXS_API int ausaxs_gpu_server_histogram(ausaxs_gpu_server* s, int32_t id, ausaxs_hist_result* out);

/*
 * Weighted linear least squares of a model against data plus chi-square, on the device:
 * fitter::detail::LinearLeastSquares::fit (source/core/fitter/detail/LinearLeastSquares.cpp:26-55),
 * fitting model ~ a * data + b with weights 1/err^2 as LinearFitter sets it up (the measured
 * intensities as data, the model on the measured q as model; source/core/fitter/LinearFitter.cpp:14-21).
 * Host pointers; out[5] = {a, b, sigma_a, sigma_b, chi2}.
 */
AUSAXS_API int ausaxs_gpu_linear_lsq(ausaxs_gpu_ctx* ctx, const double* data, const double* model, const double* err,
                                     int32_t n, double* out);

/*
 * Allocation-free Simple (weighted) histogram.  No counterpart in the reference: it exists for
 * callers that cannot allocate device memory while they run (a memory-pool-managed or real-time
 * section, or an embedding application that forbids cudaMalloc after start-up, since allocation can
 * synchronise the device).  It computes what ausaxs_gpu_histogram returns for AUSAXS_MANAGER_MT, but
 * from device inputs into device outputs, and calls no cudaMalloc, cudaFree or allocating library
 * routine: its temporaries live in one file-scope device array (591,104 bytes, about 577 KiB, per
 * device, held until the process exits).
 *   atoms, waters   : device arrays of n x {float x, y, z, w} (weights in the 4th word)
 *   bin_count       : at most 8192 (AUSAXS_ERR_CAPACITY above that); every pair distance must fall
 *                     below bin_count * bin_width.  The pair kernel keeps bin_count bins on chip, so
 *                     pass the smallest bin_count that covers the structure's largest distance: at
 *                     8,000 bins one CTA fits per SM and the call runs slower than ausaxs_gpu_histogram,
 *                     which trims its bins to the structure
 *   hist_out        : device, 5 * bin_count doubles: rows {aa, aw, ww, tot, d_axis}, each with stride
 *                     bin_count, zero beyond *max_bin_out
 *   max_bin_out     : device int32
 *   overflow_out    : device u64 (may be NULL): pairs that fell beyond bin_count
 *   stream          : cudaStream_t as void* (NULL = legacy default stream); the call only enqueues.
 * All calls share the one scratch array, which keeps the last call's contents (each call clears
 * what must start at zero); calls that overlap on the GPU race and give wrong results: issue them on
 * one stream, or order them with events.  The array's address belongs to the CUDA context: the first
 * call in each context of a device (a context created again after cudaDeviceReset is a new one)
 * looks it up and caches it, so make that first call before any stream capture.
 */
AUSAXS_API int ausaxs_gpu_histogram_mt_noalloc(const float* atoms, int32_t n_atoms, const float* waters,
                                               int32_t n_waters, double bin_width, int32_t bin_count,
                                               int32_t weighted_bins, double* hist_out, int32_t* max_bin_out,
                                               unsigned long long* overflow_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AUSAXS_B200_H */
