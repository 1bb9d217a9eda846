/*
 * CPU restatement of the AUSAXS Debye hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA path: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  It restates, in plain C and in
 * the reference's operation order, the functions listed below; each cites the
 * reference file:line it follows.  Its own correctness is pinned against the
 * reference compiled from source (oracle/_ref, see oracle/Makefile) and
 * against the reference's known-answer tests (tests/golden/).
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared (no fast-math: the pair
 * distance must be evaluated with the reference's SIMD rounding sequence).
 *
 * Conventions
 *   point     : 4 x 32-bit {x, y, z, w|ff} exactly as the reference's
 *               CompactCoordinatesXYZW / XYZFF records
 *               (include/core/hist/detail/data/CompactCoordinatesXYZW.h:131-134).
 *   ff types  : the reference's form_factor_t enum values (0 = excluded volume,
 *               1 = water/OH, ...), max 15 (include/core/form_factor/FormFactorType.h:14-37).
 *   histograms: row-major FP64 [rows][nbins].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define NFF 15 /* settings::form_factor::max_ff_types (include/core/settings/FormFactorSettings.h:12) */

typedef struct {
    float x, y, z;
    union {
        float w;
        int32_t ff;
    } v;
} opoint;

/* ---------------------------------------------------------------------------
 * Pair evaluation.
 * SIMD evaluators (CompactCoordinatesXYZW.h:382-423, :491-535, :602-655):
 *   d2 = (dx*dx + dy*dy) + dz*dz, d = sqrt(d2), bin = cvt_rn(d * inv_w)
 * with each operation rounded separately and ties to even (the squares are
 * formed before the lane shuffles, so no contraction is possible).
 * Scalar tail evaluator (CompactCoordinatesXYZW.h:303-307, IntrinsicHelpers.h:9-14):
 * dx*dx + dy*dy + dz*dz under the reference's release flags
 * (-O3 -ffast-math -march=x86-64-v3, cmake/setup_compile_commands.cmake:100-103)
 * is contracted by GCC to fma(dz, dz, fma(dx, dx, dy*dy)) -- established by
 * compiling that helper with those flags and comparing all candidate
 * contractions on 1e6 random pairs -- and bin = std::round(inv_w * d), ties
 * away from zero.
 * ------------------------------------------------------------------------- */
static inline float pair_distance(const opoint* a, const opoint* b, int tail) {
    float dx = a->x - b->x, dy = a->y - b->y, dz = a->z - b->z;
    if (tail) return sqrtf(fmaf(dz, dz, fmaf(dx, dx, dy * dy)));
    float sx = dx * dx, sy = dy * dy, sz = dz * dz;
    return sqrtf((sx + sy) + sz);
}

static inline int32_t pair_bin(float d, float inv_w, int tail) {
    float x = d * inv_w;
    return tail ? (int32_t)roundf(x) : (int32_t)rintf(x);
}

/* The j-loops of every reference driver are unrolled 16/8/4 and finish with
 * single evaluations (SimpleCalculator.h:117-141, HistogramManagerMTFFAvg.cpp:216-232):
 * the last (len mod 4) partners of a row go through the scalar evaluator. */
static inline int32_t tail_start(int32_t j0, int32_t n) { return n - ((n - j0) & 3); }

/* Row selection for one pair, by the histogram shape the reference increments. */
enum {
    ROW_SINGLE = 0, /* 1D histogram (ww, xx, wx, Simple)                               */
    ROW_FFPAIR = 1, /* [ff_i][ff_j]  (increment_linear_index, CompactCoordinatesXYZFF.h:187-188) */
    ROW_FFOUTER = 2 /* [ff_i]        (aw / ax by the outer atom's type)                */
};

typedef struct {
    double* counts; /* [rows][nbins]: += factor per pair                                 */
    double* dsum;   /* [nbins]: += factor * d (the bin_center sums of the rows that feed */
                    /*          the weighted d-axis)                                     */
    double* dcnt;   /* [nbins]: += factor (their counts)                                 */
    double* wsum;   /* [nbins] or NULL: += factor * (w_i * w_j) (XYZW weights)           */
    int64_t overflow;
} job_out;

/*
 * One pair-binning pass.  Outer set A (index i), inner set B (index j).
 * self != 0: A == B and only j > i is visited (SimpleCalculator.h:117-141).
 * FFAvg also increments the excluded-volume rows of every atom-atom pair
 * (HistogramManagerMTFFAvg.cpp:27-35): exv_rows = 2 adds [ff_i][exv] and
 * [exv][exv]; for atom-water pairs exv_rows = 1 adds [exv] (:111-117).
 */
static void pair_job(const opoint* A, int32_t na, const opoint* B, int32_t nb, int self, int row_mode, int exv_rows,
                     double factor, float inv_w, int32_t nbins, job_out* o) {
    for (int32_t i = 0; i < na; ++i) {
        int32_t j0 = self ? i + 1 : 0;
        int32_t ts = tail_start(j0, nb);
        for (int32_t j = j0; j < nb; ++j) {
            const int tail = j >= ts;
            float d = pair_distance(&A[i], &B[j], tail);
            int32_t bin = pair_bin(d, inv_w, tail);
            if (!(bin >= 0 && bin < nbins)) {
                o->overflow++;
                continue;
            }
            int32_t row = 0;
            if (row_mode == ROW_FFPAIR) row = A[i].v.ff * NFF + B[j].v.ff;
            else if (row_mode == ROW_FFOUTER) row = A[i].v.ff;
            o->counts[(size_t)row * nbins + bin] += factor;
            if (exv_rows == 2) {
                o->counts[(size_t)(A[i].v.ff * NFF + 0) * nbins + bin] += factor;
                o->counts[(size_t)0 * nbins + bin] += factor;
            } else if (exv_rows == 1) {
                o->counts[(size_t)0 * nbins + bin] += factor;
            }
            /* WeightedEntry::add/increment: bin_center += N*distance with N*distance in
             * float (include/core/hist/distribution/detail/WeightedEntry.h:63-81). */
            if (o->dsum) {
                o->dsum[bin] += (double)((float)factor * d);
                o->dcnt[bin] += factor;
            }
            if (o->wsum) o->wsum[bin] += factor * (double)(A[i].v.w * B[j].v.w);
        }
    }
}

/* ---------------------------------------------------------------------------
 * Manager post-processing helpers.
 * ------------------------------------------------------------------------- */

/* max_bin: last bin >= 10 whose total is non-zero, +1; minimum 10
 * (HistogramManagerMT.cpp:47-58, HistogramManagerMTFFAvg.cpp:339-346). */
static int32_t find_max_bin(const double* tot, int32_t nbins) {
    for (int32_t i = nbins - 1; i >= 10; --i)
        if (tot[i] != 0) return i + 1;
    return 10;
}

/* WeightedDistribution1D::get_weighted_axis (source/core/hist/distribution/WeightedDistribution1D.cpp:51-58):
 * mean distance of each bin, or the bin's lower value i*width when empty. */
static void weighted_axis(const double* dsum, const double* dcnt, int32_t n, double bin_width, double* out) {
    double w = ((double)n * bin_width) / n; /* Axis(0, n*bin_width, n).width() */
    for (int32_t i = 0; i < n; ++i) {
        double dv = 0 + i * w;
        double bc = dsum[i];
        uint32_t c = (uint32_t)dcnt[i];
        out[i] = ((double)(bc == 0) * dv + bc) / (double)((c == 0) + c);
    }
}

/*
 * HistogramManagerMT<weighted_bins, vbw>::calculate_all (source/core/hist/histogram_manager/HistogramManagerMT.cpp:23-75)
 * over SimpleCalculator (include/core/hist/distance_calculator/SimpleCalculator.h:94-215):
 * aa self (factor 2), ww self (factor 2), aw cross with waters outer / atoms inner (factor 2),
 * diagonal sum(w*w) into bin 0, truncation, and the weighted axis of p_tot.
 *
 * Outputs (first *max_bin entries used, capacity nbins): aa, aw, ww, tot = weighted counts;
 * d_axis = weighted bin centres (or i*width when !weighted), d_axis[0] = 0.
 * Returns the number of pairs whose bin fell outside [0, nbins).
 */
int64_t oracle_hist_simple(const opoint* atoms, int32_t na, const opoint* waters, int32_t nw, double bin_width,
                           int32_t nbins, int weighted, int32_t* max_bin, double* aa, double* aw, double* ww,
                           double* tot, double* d_axis) {
    float inv_w = (float)(1.0 / bin_width);
    size_t nbytes = sizeof(double) * (size_t)nbins;
    double *ca = calloc(nbins, 8), *cw = calloc(nbins, 8), *cx = calloc(nbins, 8);
    double *da = calloc(nbins, 8), *dw = calloc(nbins, 8), *dx = calloc(nbins, 8);
    double *na_ = calloc(nbins, 8), *nw_ = calloc(nbins, 8), *nx_ = calloc(nbins, 8);
    double *wa = calloc(nbins, 8), *ww_ = calloc(nbins, 8), *wx = calloc(nbins, 8);
    job_out oa = {ca, da, na_, wa, 0}, ow = {cw, dw, nw_, ww_, 0}, ox = {cx, dx, nx_, wx, 0};
    pair_job(atoms, na, atoms, na, 1, ROW_SINGLE, 0, 2.0, inv_w, nbins, &oa);
    pair_job(waters, nw, waters, nw, 1, ROW_SINGLE, 0, 2.0, inv_w, nbins, &ow);
    pair_job(waters, nw, atoms, na, 0, ROW_SINGLE, 0, 2.0, inv_w, nbins, &ox);
    /* self-correlation: scaling * sum(float(w*w)) (SimpleCalculator.h:146-160) */
    double twa = 0, tww = 0;
    for (int32_t i = 0; i < na; ++i) twa += atoms[i].v.w * atoms[i].v.w;
    for (int32_t i = 0; i < nw; ++i) tww += waters[i].v.w * waters[i].v.w;
    wa[0] += twa;
    ww_[0] += tww;
    na_[0] += (double)(uint32_t)twa;
    nw_[0] += (double)(uint32_t)tww;
    double* ptot = calloc(nbins, 8);
    double* pdsum = calloc(nbins, 8);
    double* pdcnt = calloc(nbins, 8);
    for (int32_t b = 0; b < nbins; ++b) {
        ptot[b] = wa[b] + ww_[b] + wx[b];
        pdsum[b] = da[b] + dw[b] + dx[b];
        pdcnt[b] = (double)((uint32_t)na_[b] + (uint32_t)nw_[b] + (uint32_t)nx_[b]);
    }
    int32_t mb = find_max_bin(ptot, nbins);
    *max_bin = mb;
    memcpy(aa, wa, sizeof(double) * mb);
    memcpy(aw, wx, sizeof(double) * mb);
    memcpy(ww, ww_, sizeof(double) * mb);
    memcpy(tot, ptot, sizeof(double) * mb);
    if (weighted) {
        weighted_axis(pdsum, pdcnt, mb, bin_width, d_axis);
    } else {
        double w = ((double)mb * bin_width) / mb;
        for (int32_t i = 0; i < mb; ++i) d_axis[i] = i * w;
    }
    d_axis[0] = 0; /* DistanceHistogram::initialize (DistanceHistogram.cpp:44-47) */
    int64_t of = oa.overflow + ow.overflow + ox.overflow;
    (void)nbytes;
    free(ca); free(cw); free(cx); free(da); free(dw); free(dx);
    free(na_); free(nw_); free(nx_); free(wa); free(ww_); free(wx);
    free(ptot); free(pdsum); free(pdcnt);
    return of;
}

/*
 * One job of hist::distance_calculator::SimpleCalculator<weighted_bins = true>
 * (include/core/hist/distance_calculator/SimpleCalculator.h:94-215) with a scaling factor:
 *   self (b == NULL): the pairs i < j of a with factor 2*scaling, plus the diagonal
 *        scaling * sum(float(w*w)) in bin 0 (its count: that value truncated to unsigned);
 *   cross: enqueue_calculate_cross(a, b): b outer, a inner, factor 2*scaling.
 * Accumulates value (weights), count and dsum (bin-centre sums) into the caller's arrays (nbins
 * each).  Returns the pairs whose bin fell outside [0, nbins).
 */
int64_t oracle_calc_job(const opoint* a, int32_t na, const opoint* b, int32_t nb, int32_t scaling, double bin_width,
                        int32_t nbins, double* value, double* count, double* dsum) {
    float inv_w = (float)(1.0 / bin_width);
    double* cnt = calloc(nbins, 8);
    job_out o = {cnt, dsum, count, value, 0};
    if (b == NULL) {
        pair_job(a, na, a, na, 1, ROW_SINGLE, 0, 2.0 * scaling, inv_w, nbins, &o);
        double tw = 0;
        for (int32_t i = 0; i < na; ++i) tw += a[i].v.w * a[i].v.w;
        tw *= scaling;
        value[0] += tw;
        count[0] += (double)(uint32_t)tw;
    } else {
        pair_job(b, nb, a, na, 0, ROW_SINGLE, 0, 2.0 * scaling, inv_w, nbins, &o);
    }
    free(cnt);
    return o.overflow;
}

/*
 * Form-factor managers.
 *   kind 0: HistogramManagerMTFFAvg     (source/core/hist/histogram_manager/HistogramManagerMTFFAvg.cpp:194-372)
 *   kind 1: HistogramManagerMTFFExplicit (HistogramManagerMTFFExplicit.cpp:216-437)
 *   kind 2: HistogramManagerMTFFGrid     (HistogramManagerMTFFGrid.cpp:43-234): FFAvg plus the
 *           excluded-volume dummies exv[] (ax, wx, xx) replacing the exv rows.
 * Atoms must carry ff >= 1.  Outputs (capacity nbins, first *max_bin used per row):
 *   aa [15][15][mb], aw [15][mb], ww [mb], tot [mb] (p_tot counts), d_axis [mb];
 *   for kind 2 also d_axis_ax, d_axis_xx [mb].
 * z_exv: the average excluded-volume charge V_grid * rho_w / N_atoms (kind 0 only).
 */
int64_t oracle_hist_ff(int kind, const opoint* atoms, int32_t na, const opoint* waters, int32_t nw, const opoint* exv,
                       int32_t nx, double bin_width, int32_t nbins, double z_exv, int32_t* max_bin, double* aa,
                       double* aw, double* ww, double* tot, double* d_axis, double* d_axis_ax, double* d_axis_xx) {
    float inv_w = (float)(1.0 / bin_width);
    size_t nb = (size_t)nbins;
    double* caa = calloc(NFF * NFF * nb, 8);
    double* caw = calloc(NFF * nb, 8);
    double* cww = calloc(nb, 8);
    double* dsum = calloc(nb, 8);
    double* dcnt = calloc(nb, 8);
    /* FFExplicit has no exv rows (HistogramManagerMTFFExplicit.cpp:27-35 increments only [ff_i][ff_j]) */
    int exv_aa = kind == 1 ? 0 : 2, exv_aw = kind == 1 ? 0 : 1;
    job_out o1 = {caa, dsum, dcnt, NULL, 0};
    pair_job(atoms, na, atoms, na, 1, ROW_FFPAIR, exv_aa, 2.0, inv_w, nbins, &o1);
    job_out o2 = {caw, dsum, dcnt, NULL, 0};
    pair_job(atoms, na, waters, nw, 0, ROW_FFOUTER, exv_aw, 1.0, inv_w, nbins, &o2);
    job_out o3 = {cww, dsum, dcnt, NULL, 0};
    pair_job(waters, nw, waters, nw, 1, ROW_SINGLE, 0, 2.0, inv_w, nbins, &o3);
    int64_t of = o1.overflow + o2.overflow + o3.overflow;

    /* self-correlations (HistogramManagerMTFFAvg.cpp:310-323) */
    for (int32_t i = 0; i < na; ++i) {
        int32_t f = atoms[i].v.ff;
        caa[(size_t)(f * NFF + f) * nb + 0] += 1;
        dcnt[0] += 1;
    }
    if (kind != 1) caa[0] += na; /* [exv][exv][0] += N_a, not part of p_tot */
    cww[0] += nw;
    dcnt[0] += nw;

    /* p_tot = sum over ff >= 1 of aa and aw, plus ww (HistogramManagerMTFFAvg.cpp:325-337) */
    double* ptot = calloc(nb, 8);
    for (int f1 = 1; f1 < NFF; ++f1)
        for (int f2 = 1; f2 < NFF; ++f2)
            for (size_t b = 0; b < nb; ++b) ptot[b] += caa[(size_t)(f1 * NFF + f2) * nb + b];
    for (int f1 = 1; f1 < NFF; ++f1)
        for (size_t b = 0; b < nb; ++b) ptot[b] += caw[(size_t)f1 * nb + b];
    for (size_t b = 0; b < nb; ++b) ptot[b] += cww[b];
    int32_t mb = find_max_bin(ptot, nbins);

    if (kind == 0) {
        /* Z_exv scaling of the exv rows (HistogramManagerMTFFAvg.cpp:355-364) */
        for (int f1 = 1; f1 < NFF; ++f1)
            for (int32_t b = 0; b < mb; ++b) caa[(size_t)(f1 * NFF + 0) * nb + b] *= z_exv;
        /* val * (Z * Z): the reference release build (-ffast-math) hoists Z*Z out of the loop of
         * HistogramManagerMTFFAvg.cpp:361-362; checked against its output (tests/golden) */
        for (int32_t b = 0; b < mb; ++b) caa[b] *= z_exv * z_exv;
        for (int32_t b = 0; b < mb; ++b) caw[b] *= z_exv;
    }

    if (kind == 2) {
        /* grid excluded volume (HistogramManagerMTFFGrid.cpp:68-233) */
        double* cax = calloc(NFF * nb, 8);
        double* cwx = calloc(nb, 8);
        double* cxx = calloc(nb, 8);
        double* dax = calloc(nb, 8);
        double* nax = calloc(nb, 8);
        double* dxx = calloc(nb, 8);
        double* nxx = calloc(nb, 8);
        job_out ox = {cxx, dxx, nxx, NULL, 0};
        pair_job(exv, nx, exv, nx, 1, ROW_SINGLE, 0, 2.0, inv_w, nbins, &ox);
        job_out oax = {cax, dax, nax, NULL, 0};
        pair_job(atoms, na, exv, nx, 0, ROW_FFOUTER, 0, 1.0, inv_w, nbins, &oax);
        job_out owx = {cwx, dax, nax, NULL, 0};
        pair_job(waters, nw, exv, nx, 0, ROW_SINGLE, 0, 1.0, inv_w, nbins, &owx);
        of += ox.overflow + oax.overflow + owx.overflow;
        cxx[0] += nx;
        nxx[0] += nx;
        int32_t mbx = 10;
        for (int32_t i = nbins - 1; i >= 10; --i)
            if (cxx[i] != 0 || cwx[i] != 0) {
                mbx = i + 1;
                break;
            }
        if (mbx > mb) mb = mbx;
        for (int f1 = 0; f1 < NFF; ++f1)
            for (int32_t b = 0; b < mb; ++b) caa[(size_t)(f1 * NFF + 0) * nb + b] = cax[(size_t)f1 * nb + b];
        for (int32_t b = 0; b < mb; ++b) caw[b] = cwx[b];
        for (int32_t b = 0; b < mb; ++b) caa[b] = cxx[b];
        /* ax / xx axes keep their weighted value in bin 0 (CompositeDistanceHistogramFFGrid.cpp:129-134) */
        weighted_axis(dax, nax, mb, bin_width, d_axis_ax);
        weighted_axis(dxx, nxx, mb, bin_width, d_axis_xx);
        free(cax); free(cwx); free(cxx); free(dax); free(nax); free(dxx); free(nxx);
    }

    *max_bin = mb;
    for (int r = 0; r < NFF * NFF; ++r) memcpy(aa + (size_t)r * mb, caa + (size_t)r * nb, sizeof(double) * mb);
    for (int r = 0; r < NFF; ++r) memcpy(aw + (size_t)r * mb, caw + (size_t)r * nb, sizeof(double) * mb);
    memcpy(ww, cww, sizeof(double) * mb);
    memcpy(tot, ptot, sizeof(double) * mb);
    weighted_axis(dsum, dcnt, mb, bin_width, d_axis);
    d_axis[0] = 0;
    free(caa); free(caw); free(cww); free(dsum); free(dcnt); free(ptot);
    return of;
}

/* ---------------------------------------------------------------------------
 * Debye transform (FP64), generalised to arbitrary q.
 * ------------------------------------------------------------------------- */

/* VectorDebyeTable::initialize (source/core/table/VectorDebyeTable.cpp:24-40) */
static double sinc_ref(double qd) {
    if (qd < 1e-3) {
        double qd2 = qd * qd;
        return 1 - qd2 * (1.0 / 6) + qd2 * qd2 * (1.0 / 120);
    }
    return sin(qd) / qd;
}

/* sinqd[r][q] = sum_b p[r][b] * sinc(q * d[b])  (std::inner_product order,
 * CompositeDistanceHistogramFFAvgBase.cpp:427-467) */
void oracle_sinqd(const double* p, int32_t rows, int32_t nbins, const double* d_axis, const double* q, int32_t nq,
                  double* out) {
    double* s = malloc(sizeof(double) * (size_t)nbins);
    for (int32_t k = 0; k < nq; ++k) {
        for (int32_t b = 0; b < nbins; ++b) s[b] = sinc_ref(q[k] * d_axis[b]);
        for (int32_t r = 0; r < rows; ++r) {
            double acc = 0;
            const double* pr = p + (size_t)r * nbins;
            for (int32_t b = 0; b < nbins; ++b) acc = acc + pr[b] * s[b];
            out[(size_t)r * nq + k] = acc;
        }
    }
    free(s);
}

/* Five-Gaussian atomic form factors: f(q) = sum_i a_i exp(-b_i q^2) + c, with
 * b given in s = q/(4 pi) units and converted by 1/(16 pi^2)
 * (include/core/form_factor/FormFactorTable.h:8-21, FormFactor.h:33-39).
 * Coefficients: Waasmaier & Kirfel (1995) for C, N, O, S and argon (OTHER);
 * International Tables for H; Grudinin, Garkavenko & Kazennov (2017) for the
 * united-atom groups (FormFactorTable.h:24-186).  Index = form_factor_t. */
typedef struct {
    double a[5], b[5], c;
} ff5;

static const ff5 FF_TABLE[NFF] = {
    /* 0 EXCLUDED_VOLUME: a={1}, b={r^2/2} with r = 1.62 (FormFactorTable.h, excluded_volume) */
    {{1, 0, 0, 0, 0}, {-1, 0, 0, 0, 0}, 0},
    /* 1 WATER = OH (OH_alc) */
    {{0.456221, 3.219608, 0.812773, 2.666928, 1.380927}, {21.503498, 13.397134, 34.547137, 5.826620, 0.412902}, 0.463202},
    /* 2 H */
    {{0.489918, 0.262003, 0.196767, 0.049879, 0}, {20.6593, 7.74039, 49.5519, 2.20159, 0}, 0.001305},
    /* 3 C */
    {{2.657506, 1.078079, 1.490909, -4.241070, 0.713791}, {14.780758, 0.776775, 42.086843, -0.000294, 0.239535}, 4.297983},
    /* 4 CH (CH_sp3) */
    {{2.909530, 0.485267, 1.516151, 0.206905, 1.541626}, {13.933084, 23.221524, 41.990403, 4.974183, 0.679266}, 0.337670},
    /* 5 CH2 (CH2_sp3) */
    {{3.275723, 0.870037, 1.534606, 0.395078, 1.544562}, {13.408502, 23.785175, 41.922444, 5.019072, 0.724439}, 0.377096},
    /* 6 CH3 (CH3_sp3) */
    {{3.681341, 1.228691, 1.549320, 0.574033, 1.554377}, {13.026207, 24.131974, 41.869426, 4.984373, 0.765769}, 0.409294},
    /* 7 N */
    {{11.893780, 3.277479, 1.858092, 0.858927, 0.912985}, {0.000158, 10.232723, 30.344690, 0.656065, 0.217287}, -11.804902},
    /* 8 NH */
    {{1.650531, 0.429639, 2.144736, 1.851894, 1.408921}, {10.603730, 6.987283, 29.939901, 10.573859, 0.611678}, 0.510589},
    /* 9 NH2 */
    {{1.904157, 1.942536, 2.435585, 0.730512, 1.379728}, {10.803702, 10.792421, 29.610479, 6.847755, 0.709687}, 0.603738},
    /* 10 NH3 (NH3_plus) */
    {{1.882162, 1.933200, 2.465843, 0.927311, 1.190889}, {10.975157, 10.956008, 29.208572, 6.663555, 0.843650}, 0.597322},
    /* 11 O */
    {{2.960427, 2.508818, 0.637853, 0.722838, 1.142756}, {14.182259, 5.936858, 0.112726, 34.958481, 0.390240}, 0.027014},
    /* 12 S */
    {{6.362157, 5.154568, 1.473732, 1.635073, 1.209372}, {1.514347, 22.092528, 0.061373, 55.445176, 0.646925}, 0.154722},
    /* 13 SH */
    {{0.570042, 6.337416, 1.641643, 5.398549, 1.527982}, {11.447986, 1.197657, 55.401032, 22.420955, 2.356552}, 1.523944},
    /* 14 OTHER (argon) */
    {{7.188004, 6.638454, 0.454180, 1.929593, 1.523654}, {0.956221, 15.339877, 15.339862, 39.043824, 0.062409}, 0.265954},
};

static const double PI_ = 3.14159265358979323846;

/* raw FormFactor::evaluate(q) with q0 = 1 (FormFactor.h:33-39) */
double oracle_ff_raw(int type, double q) {
    const ff5* f = &FF_TABLE[type];
    double s_to_q = 1. / (4 * 4 * PI_ * PI_);
    double sum = 0;
    for (int i = 0; i < 5; ++i) {
        double b = (type == 0) ? (i == 0 ? 1.62 * 1.62 / 2 : 0) : f->b[i] * s_to_q;
        sum += f->a[i] * exp(-b * q * q);
    }
    return sum + f->c;
}

/* ExvFormFactor(V).evaluate(q) = V rho_w exp(-V^(2/3)/(4 pi) q^2)
 * (include/core/form_factor/ExvFormFactor.h:20-33), rho_w = 0.334 e/A^3 (Constants.h:114) */
double oracle_ff_exv_volume(double volume, double q) {
    double e = pow(volume, 2. / 3) / (4 * PI_);
    return volume * 0.334 * exp(-e * q * q);
}

/* Excluded volume per form_factor_t of the reference's default set for explicit excluded volume,
 * constants::exv::MinimumFluctuation_implicit_H (include/core/form_factor/ExvTable.h:67-81; OTHER
 * uses the argon sphere, 4 pi/3 * 1.88^3, ExvTable.h:135 and vdwTable.h:13), in the order of
 * ExvFormFactorSet::get (include/core/form_factor/ExvFormFactor.h:53-72).  Entry 0 is unused. */
double oracle_exv_volume(int type) {
    static const double v[NFF] = {0.0,    20.911, 0.0,    12.352, 11.640, 34.583, 41.851, 0.027,
                                  2.181,  20.562, 20.722, 14.238, 15.413, 28.529, 0.0};
    if (type == NFF - 1) return 4 * PI_ / 3 * 1.88 * 1.88 * 1.88;
    return (type >= 0 && type < NFF) ? v[type] : 0.0;
}

/*
 * FFAvg / FFGrid / FFExplicit intensity (CompositeDistanceHistogramFFAvgBase.cpp:57-76, 333-374, 470-558;
 * CompositeDistanceHistogramFFGrid.cpp:37-119).
 *   kind 0 (FFAvg): products of raw form factors, F(ff, exv) uses the raw excluded_volume entry.
 *   kind 2 (FFGrid): F(ff, exv) = f_ff * ExvFormFactor(width^3), F(exv, exv) likewise, and ax/wx
 *                    use d_axis_ax, xx uses d_axis_xx.
 *   kind 1 (FFExplicit, CompositeDistanceHistogramFFExplicitBase.cpp:54-57, 64-211): the atom-atom
 *                    and atom-water sinc sums serve aa/ax/xx and aw/wx with per-type excluded-volume
 *                    form factors x_t = ExvFormFactor(V_t); ax += crho e(q) s_aa[f1][f2]
 *                    (f_f1 x_f2 + f_f2 x_f1), xx += (e(q) crho)^2 s_aa[f1][f2] x_f1 x_f2,
 *                    wx += crho e(q) cw s_aw[f1] (f_w x_f1 + f_f1 x_w), with
 *                    e(q) = cx^3 exp(-(1.62^2/4)(cx^2 - 1) q^2) in place of cx.
 * Inputs: the histograms as returned by oracle_hist_ff (mb bins).  Outputs profiles[6][nq]
 * = {aa, ax, aw, xx, wx, ww} and Iq = aa - ax + aw + xx - wx + ww.
 */
/* The sinc sums of every raw histogram row (they do not depend on cw, cx, crho or the Debye-Waller
 * factors; the reference caches them the same way, CompositeDistanceHistogramFFAvgBase.cpp:377-397). */
typedef struct {
    double* s_aa; /* [15][15][nq] */
    double* s_aw; /* [15][nq] */
    double* s_ww; /* [nq] */
} ff_sums;

static void ff_sums_compute(int kind, const double* aa, const double* aw, const double* ww, int32_t mb,
                            const double* d_axis, const double* d_axis_ax, const double* d_axis_xx, const double* q,
                            int32_t nq, ff_sums* S) {
    S->s_aa = malloc(sizeof(double) * (size_t)NFF * NFF * nq);
    S->s_aw = malloc(sizeof(double) * (size_t)NFF * nq);
    S->s_ww = malloc(sizeof(double) * (size_t)nq);
    const double* dax = kind == 2 ? d_axis_ax : d_axis;
    const double* dxx = kind == 2 ? d_axis_xx : d_axis;
    /* aa rows: ff1 >= 1 and ff2 >= 1 with the aa axis; [ff][exv] with the ax axis; [exv][exv] with xx */
    for (int f1 = 0; f1 < NFF; ++f1) {
        for (int f2 = 0; f2 < NFF; ++f2) {
            const double* ax = (f1 == 0 && f2 == 0) ? dxx : (f2 == 0 ? dax : d_axis);
            oracle_sinqd(aa + (size_t)(f1 * NFF + f2) * mb, 1, mb, ax, q, nq, S->s_aa + (size_t)(f1 * NFF + f2) * nq);
        }
        oracle_sinqd(aw + (size_t)f1 * mb, 1, mb, f1 == 0 ? dax : d_axis, q, nq, S->s_aw + (size_t)f1 * nq);
    }
    oracle_sinqd(ww, 1, mb, d_axis, q, nq, S->s_ww);
}

static void ff_sums_free(ff_sums* S) {
    free(S->s_aa);
    free(S->s_aw);
    free(S->s_ww);
}

/* The profiles and I(q) from the sinc sums and the free parameters. */
static void ff_combine(int kind, const ff_sums* S, const double* q, int32_t nq, double cw, double cx, double crho,
                       double dw_atomic, double dw_exv, double grid_width, double* profiles, double* Iq) {
    const double* s_aa = S->s_aa;
    const double* s_aw = S->s_aw;
    const double* s_ww = S->s_ww;
    double Vg = grid_width * grid_width * grid_width;
    for (int32_t k = 0; k < nq; ++k) {
        double qq = q[k];
        double fa[NFF];
        for (int t = 0; t < NFF; ++t) fa[t] = oracle_ff_raw(t, qq);
        double fx = kind == 2 ? oracle_ff_exv_volume(Vg, qq) : fa[0];
        double paa = 0, pax = 0, paw = 0, pxx = 0, pwx = 0, pww = 0;
        for (int f1 = 1; f1 < NFF; ++f1)
            for (int f2 = 1; f2 < NFF; ++f2) paa += s_aa[(size_t)(f1 * NFF + f2) * nq + k] * (fa[f1] * fa[f2]);
        if (kind == 1) {
            const double rm2 = 1.62 * 1.62 / 4;
            double e = pow(cx, 3) * exp(-rm2 * (pow(cx, 2) - 1) * qq * qq);
            double xe[NFF];
            for (int t = 0; t < NFF; ++t) xe[t] = oracle_ff_exv_volume(oracle_exv_volume(t), qq);
            for (int f1 = 1; f1 < NFF; ++f1)
                for (int f2 = 1; f2 < NFF; ++f2) {
                    double s = s_aa[(size_t)(f1 * NFF + f2) * nq + k];
                    pax += crho * e * s * (fa[f1] * xe[f2] + fa[f2] * xe[f1]);
                    pxx += pow(e * crho, 2) * s * (xe[f1] * xe[f2]);
                }
            for (int f1 = 1; f1 < NFF; ++f1) {
                double s = s_aw[(size_t)f1 * nq + k];
                paw += 2 * cw * s * (fa[f1] * fa[1]);
                pwx += crho * e * cw * s * (fa[1] * xe[f1] + fa[f1] * xe[1]);
            }
            pww = cw * cw * s_ww[k] * (fa[1] * fa[1]);
        } else {
            double cxq = cx; /* exv_factor(q) = cx for FFAvg / FFGrid */
            for (int f1 = 1; f1 < NFF; ++f1) pax += 2 * crho * cxq * s_aa[(size_t)(f1 * NFF + 0) * nq + k] * (fa[f1] * fx);
            pxx = pow(cxq * crho, 2) * s_aa[k] * (fx * fx);
            for (int f1 = 1; f1 < NFF; ++f1) paw += 2 * cw * s_aw[(size_t)f1 * nq + k] * (fa[f1] * fa[1]);
            pww = cw * cw * s_ww[k] * (fa[1] * fa[1]);
            pwx = 2 * crho * cxq * cw * s_aw[k] * (fx * fa[1]);
        }
        if (dw_atomic != 0 || dw_exv != 0) {
            double ba = exp(-qq * qq * dw_atomic * dw_atomic * 0.5);
            double bx = exp(-qq * qq * dw_exv * dw_exv * 0.5);
            paa *= ba * ba;
            pxx *= bx * bx;
            pax *= ba * bx;
            paw *= ba;
            pwx *= bx;
        }
        if (profiles) {
            profiles[0 * nq + k] = paa;
            profiles[1 * nq + k] = pax;
            profiles[2 * nq + k] = paw;
            profiles[3 * nq + k] = pxx;
            profiles[4 * nq + k] = pwx;
            profiles[5 * nq + k] = pww;
        }
        double I = 0;
        I += paa;
        I -= pax;
        I += paw;
        I += pxx;
        I -= pwx;
        I += pww;
        Iq[k] = I;
    }
}

void oracle_debye_ff(int kind, const double* aa, const double* aw, const double* ww, int32_t mb, const double* d_axis,
                     const double* d_axis_ax, const double* d_axis_xx, const double* q, int32_t nq, double cw,
                     double cx, double crho, double dw_atomic, double dw_exv, double grid_width, double* profiles,
                     double* Iq) {
    ff_sums S;
    ff_sums_compute(kind, aa, aw, ww, mb, d_axis, d_axis_ax, d_axis_xx, q, nq, &S);
    ff_combine(kind, &S, q, nq, cw, cx, crho, dw_atomic, dw_exv, grid_width, profiles, Iq);
    ff_sums_free(&S);
}

/* Simple composite intensity: exp(-q^2) * sum_b (aa + k aw + k^2 ww) sinc(q d)
 * (DistanceHistogram.cpp:54-87, CompositeDistanceHistogram.cpp:55-57). */
void oracle_debye_simple(const double* aa, const double* aw, const double* ww, int32_t mb, const double* d_axis,
                         const double* q, int32_t nq, double cw, double* Iq) {
    double* p = malloc(sizeof(double) * (size_t)mb);
    for (int32_t b = 0; b < mb; ++b) p[b] = aa[b] + cw * aw[b] + cw * cw * ww[b];
    oracle_sinqd(p, 1, mb, d_axis, q, nq, Iq);
    for (int32_t k = 0; k < nq; ++k) Iq[k] *= exp(-q[k] * q[k]);
    free(p);
}

/* fitter::detail::LinearLeastSquares::fit_params_only + chi2
 * (source/core/fitter/detail/LinearLeastSquares.cpp:26-44, :71-78):
 * fit model ~ a * data + b with weights 1/err^2.  out = {a, b, a_err, b_err, chi2}. */
void oracle_linear_lsq(const double* data, const double* model, const double* err, int32_t n, double* out) {
    double S = 0, Sx = 0, Sy = 0, Sxx = 0, Sxy = 0;
    for (int32_t i = 0; i < n; ++i) {
        double is = 1. / err[i];
        double w = is * is;
        S += w;
        Sx += data[i] * w;
        Sy += model[i] * w;
        Sxx += pow(data[i], 2) * w;
        Sxy += data[i] * model[i] * w;
    }
    double delta = S * Sxx - Sx * Sx;
    double a = (S * Sxy - Sx * Sy) / delta;
    double b = (Sxx * Sy - Sx * Sxy) / delta;
    double chi2 = 0;
    for (int32_t i = 0; i < n; ++i) {
        double r = (model[i] - (a * data[i] + b)) * (1. / err[i]);
        chi2 += r * r;
    }
    out[0] = a;
    out[1] = b;
    out[2] = S / delta;
    out[3] = Sxx / delta;
    out[4] = chi2;
}

/*
 * fitter::SmartFitter::fit() with one enabled parameter and the minimiser of a build without dlib,
 * mini::Golden (source/core/fitter/SmartFitter.cpp:147-176, source/core/mini/Golden.cpp:26-74), for
 * data on the model's own q axis (SmartFitter::splice then returns the model values).
 *   kind: 0 FFAvg, 1 FFExplicit, 2 FFGrid (histograms as oracle_debye_ff), 3 Simple (aa, aw, ww
 *         weighted counts, only param 0 applies);
 *   param: 0 cw, 1 cx, 2 crho, 3 dw_atomic, 4 dw_exv searched in [lo, hi] to an interval of width
 *         tol (mini::Minimizer::tol); base[5]: the other parameters' values;
 *   out = {value (centre of the final interval), a, b, chi2 at value, function evaluations as the
 *         reference reports them (without the final evaluation at value)}.
 * Each evaluation is the reference's: the transform at the trial parameters, then the linear fit
 * data ~ a * model + b with weights 1/sigma^2 and chi2 = sum ((data - (a model + b)) / sigma)^2.
 */
typedef struct {
    int kind;
    const ff_sums* S;
    const double *aa, *aw, *ww, *d_axis, *q, *y, *sigma;
    int32_t mb, nq;
    int param;
    double par[5], grid_width;
    double *I, lsq[5];
    int fevals;
} fit_ctx;

static double fit_chi2(fit_ctx* F, double v) {
    F->par[F->param] = v;
    if (F->kind == 3)
        oracle_debye_simple(F->aa, F->aw, F->ww, F->mb, F->d_axis, F->q, F->nq, F->par[0], F->I);
    else
        ff_combine(F->kind, F->S, F->q, F->nq, F->par[0], F->par[1], F->par[2], F->par[3], F->par[4], F->grid_width,
                   NULL, F->I);
    oracle_linear_lsq(F->I, F->y, F->sigma, F->nq, F->lsq);
    F->fevals += 1;
    return F->lsq[4];
}

void oracle_fit(int kind, const double* aa, const double* aw, const double* ww, int32_t mb, const double* d_axis,
                const double* d_axis_ax, const double* d_axis_xx, const double* q, const double* y,
                const double* sigma, int32_t nq, int param, double lo, double hi, double tol, const double* base,
                double grid_width, double* out) {
    ff_sums S = {0, 0, 0};
    if (kind != 3) ff_sums_compute(kind, aa, aw, ww, mb, d_axis, d_axis_ax, d_axis_xx, q, nq, &S);
    fit_ctx F;
    memset(&F, 0, sizeof F);
    F.kind = kind;
    F.S = &S;
    F.aa = aa, F.aw = aw, F.ww = ww, F.d_axis = d_axis, F.q = q, F.y = y, F.sigma = sigma;
    F.mb = mb, F.nq = nq, F.param = param, F.grid_width = grid_width;
    for (int k = 0; k < 5; ++k) F.par[k] = base[k];
    F.I = malloc(sizeof(double) * (size_t)(nq > 0 ? nq : 1));

    /* Golden::search (Golden.cpp:26-67) */
    const double phi = (1 + sqrt(5)) / 2, invphi = 1 / phi, invphi2 = invphi * invphi;
    double a = lo, b = hi, temp = a + b;
    a = fmin(a, b);
    b = temp - a;
    double diff = b - a, ilo = a, ihi = b;
    if (!(diff < tol)) {
        unsigned int n = (unsigned int)ceil(log(tol / diff) / log(invphi));
        double c = a + invphi2 * diff, d = a + invphi * diff;
        double fc = fit_chi2(&F, c), fd = fit_chi2(&F, d);
        for (unsigned int k = 0; k < n - 1; k++) {
            if (fc < fd) {
                b = d;
                d = c;
                fd = fc;
                diff = invphi * diff;
                c = a + invphi2 * diff;
                fc = fit_chi2(&F, c);
            } else {
                a = c;
                c = d;
                fc = fd;
                diff = invphi * diff;
                d = a + invphi * diff;
                fd = fit_chi2(&F, d);
            }
        }
        if (fc < fd) ilo = a, ihi = d;
        else ilo = c, ihi = b;
    }
    /* Golden::minimize_override: the interval's centre (Limit::center = min + span / 2) and its chi2 */
    const double value = ilo + (ihi - ilo) / 2;
    /* the reference reports the count taken before this last evaluation: in
       Result(p, function({p.value}), fevals) GCC reads fevals before making the call */
    out[4] = F.fevals;
    out[3] = fit_chi2(&F, value);
    out[0] = value;
    out[1] = F.lsq[0];
    out[2] = F.lsq[1];
    free(F.I);
    if (kind != 3) ff_sums_free(&S);
}

/*
 * Grid excluded-volume dummies, RawGridExv::create on the expanded molecular grid
 * (source/core/grid/exv/RawGridExv.cpp:10-59) as HistogramManagerMTFFGrid::calculate_all() sees it
 * (Molecule::get_volume_grid() expands the grid first, Grid.cpp:428-431), with the reference's
 * default settings: cell width 1 A, scaling 0.25 (1 for structures under 50 A in any direction),
 * min_exv_radius (rvol) 2.15 A, exv width 1 A, AtomicOnly expansion, hydration shell correction
 * -0.35 A (source/core/settings/GridSettings.cpp, MoleculeSettings.cpp:41).
 *   axes (Grid.cpp:34-102): the bounding box of atoms, waters and the origin, widened per axis by
 *     max(diff/2 * scaling, r_vdw(P) + r_vdw(O) + shell correction + 3 cells), floored/ceiled with
 *     one more cell; bins = (max - min) / width;
 *   members (Grid.cpp:332-375): each atom marks the cell round((x - min) / width) A_CENTER, each
 *     water W_CENTER;
 *   expansion (include/core/grid/expansion/SphericalExpander.h:27-76): for every atom, cells of the
 *     box bin +- ceil(max(r_vdw, rvol) / width) whose centre lies within r_vdw get A_AREA when they hold
 *     nothing but VOLUME, within (r_vdw, rvol] VOLUME when they hold nothing;
 *   dummies: cells with A_CENTER, A_AREA or VOLUME, swept x-major over the atoms' bin box widened by
 *     round(max(rvol, 2) / width) cells, at their centres min + i * width.
 * atoms: n x {x, y, z, ff} (double), waters: n x {x, y, z}.  Writes up to cap dummies (n x 3) and
 * returns their count; *volume = count * width^3 (Grid::get_volume).
 */
static double vdw_of_ff(int ff) {
    /* constants::radius::get_vdw_radius(form_factor_t) (include/core/form_factor/FormFactorType.h:173-192)
     * over include/core/constants/vdwTable.h: H 1.1, C 1.96, N 1.79, O 1.71, S 2.06, Ar 1.88 */
    switch (ff) {
        case 1: return 1.71;                                /* WATER = OH: oxygen */
        case 2: return 1.1;                                 /* H */
        case 3: case 4: case 5: case 6: return 1.96;        /* C, CH, CH2, CH3 */
        case 7: case 8: case 9: case 10: return 1.79;       /* N, NH, NH2, NH3 */
        case 11: return 1.71;                               /* O */
        case 12: case 13: return 2.06;                      /* S, SH */
        case 14: return 1.88;                               /* OTHER: argon */
        default: return 0.0;
    }
}

int64_t oracle_grid_exv(const double* atoms, int32_t na, const double* waters, int32_t nw, double* out, int64_t cap,
                        double* volume) {
    enum { A_CENTER = 1, W_CENTER = 2, A_AREA = 4, VOLUME = 8 };
    const double width = 1.0, rvol = 2.15;
    double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    for (int32_t i = 0; i < na; ++i)
        for (int d = 0; d < 3; ++d) {
            if (atoms[4 * (size_t)i + d] < mn[d]) mn[d] = atoms[4 * (size_t)i + d];
            if (atoms[4 * (size_t)i + d] > mx[d]) mx[d] = atoms[4 * (size_t)i + d];
        }
    for (int32_t i = 0; i < nw; ++i)
        for (int d = 0; d < 3; ++d) {
            if (waters[3 * (size_t)i + d] < mn[d]) mn[d] = waters[3 * (size_t)i + d];
            if (waters[3 * (size_t)i + d] > mx[d]) mx[d] = waters[3 * (size_t)i + d];
        }
    double diff[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    double scaling = (diff[0] < 50 || diff[1] < 50 || diff[2] < 50) ? 1.0 : 0.25;
    double margin = 2.14 + 1.71 + (-0.35) + 3 * width;
    double gmin[3];
    int bins[3];
    for (int d = 0; d < 3; ++d) {
        double e = fmax(0.5 * diff[d] * scaling, margin);
        gmin[d] = floor(mn[d] - e - width);
        double gmax = ceil(mx[d] + e + width);
        bins[d] = (int)((gmax - gmin[d]) / width);
    }
    size_t cells = (size_t)bins[0] * bins[1] * bins[2];
    unsigned char* g = calloc(cells, 1);
    if (!g) return -1;
#define CELL(i, j, k) g[((size_t)(i) * bins[1] + (j)) * bins[2] + (k)]
    int lo[3] = {1 << 30, 1 << 30, 1 << 30}, hi[3] = {-(1 << 30), -(1 << 30), -(1 << 30)};
    for (int32_t i = 0; i < na; ++i) {
        int b[3];
        for (int d = 0; d < 3; ++d) {
            b[d] = (int)round((atoms[4 * (size_t)i + d] - gmin[d]) / width);
            if (b[d] < lo[d]) lo[d] = b[d];
            if (b[d] + 1 > hi[d]) hi[d] = b[d] + 1;
        }
        CELL(b[0], b[1], b[2]) |= A_CENTER;
    }
    for (int32_t i = 0; i < nw; ++i) {
        int b[3];
        for (int d = 0; d < 3; ++d) b[d] = (int)round((waters[3 * (size_t)i + d] - gmin[d]) / width);
        CELL(b[0], b[1], b[2]) |= W_CENTER;
    }
    for (int32_t a = 0; a < na; ++a) {
        const double* p = atoms + 4 * (size_t)a;
        double rvdw = vdw_of_ff((int)p[3]), rvdw2 = rvdw * rvdw, rvol2 = rvol * rvol;
        int br = (int)ceil(fmax(rvdw, rvol) / width);
        int b[3], lo_[3], hi_[3];
        for (int d = 0; d < 3; ++d) {
            b[d] = (int)round((p[d] - gmin[d]) / width);
            lo_[d] = b[d] - br > 0 ? b[d] - br : 0;
            hi_[d] = b[d] + br + 1 < bins[d] ? b[d] + br + 1 : bins[d];
        }
        for (int i = lo_[0]; i < hi_[0]; ++i) {
            double x2 = pow(gmin[0] + i * width - p[0], 2);
            for (int j = lo_[1]; j < hi_[1]; ++j) {
                double x2y2 = x2 + pow(gmin[1] + j * width - p[1], 2);
                for (int k = lo_[2]; k < hi_[2]; ++k) {
                    double dist = x2y2 + pow(gmin[2] + k * width - p[2], 2);
                    unsigned char* c = &CELL(i, j, k);
                    int fill = dist <= rvdw2;
                    if (fill) {
                        if (!(*c == 0 || *c == VOLUME)) continue;
                        *c |= A_AREA;
                    } else if (dist <= rvol2) {
                        if (*c != 0) continue;
                        *c |= VOLUME;
                    }
                }
            }
        }
    }
    int buffer = (int)fmax(1.0, round(fmax(rvol, 2.0) / width));
    int64_t n = 0;
    if (na > 0) {
        for (int i = lo[0] - buffer > 0 ? lo[0] - buffer : 0; i < (hi[0] + buffer + 1 < bins[0] ? hi[0] + buffer + 1 : bins[0]); ++i)
            for (int j = lo[1] - buffer > 0 ? lo[1] - buffer : 0; j < (hi[1] + buffer + 1 < bins[1] ? hi[1] + buffer + 1 : bins[1]); ++j)
                for (int k = lo[2] - buffer > 0 ? lo[2] - buffer : 0; k < (hi[2] + buffer + 1 < bins[2] ? hi[2] + buffer + 1 : bins[2]); ++k) {
                    if (!(CELL(i, j, k) & (A_CENTER | A_AREA | VOLUME))) continue;
                    if (out && n < cap) {
                        out[3 * n] = gmin[0] + i * width;
                        out[3 * n + 1] = gmin[1] + j * width;
                        out[3 * n + 2] = gmin[2] + k * width;
                    }
                    ++n;
                }
    }
#undef CELL
    free(g);
    if (volume) *volume = (double)n * width * width * width;
    return n;
}

/*
 * Hydration shell, Molecule::generate_new_hydration() with the reference's default strategy:
 * RadialHydration (source/core/hydrate/generation/RadialHydration.cpp:43-206) on the grid of
 * GridBasedHydration::hydrate (GridBasedHydration.cpp:34-79), no culling (NoCulling.cpp).
 *   axes: as Grid(bodies) builds them (Grid.cpp:34-102), from the atoms alone (the hydration is
 *     cleared before the grid is made), with the box extents truncated to int: oracle_hydrate_axes;
 *   grid: each atom marks its cell A_CENTER; expand_volume() then marks, per atom, the cells within
 *     r_vdw A_AREA and those within (r_vdw, rvol] VOLUME (SphericalExpander.h:27-76);
 *   directions: prepare_rotations(8): one octant of the sphere at theta, phi in {0, pi/4, pi/2},
 *     reflected into all eight octants, components below 1e-5 zeroed and duplicates (distance
 *     < 1e-5) dropped, in first-seen order: 26 unit vectors; probe offsets round(k rh u) / width
 *     for k = 1, 3, 5, with rh = r_vdw(O) + shell correction = 1.71 - 0.35;
 *   candidates, atom by atom in grid order and direction by direction: x = atom + u (r_vdw + rh) +
 *     noise (formed as fma(u, r_vdw + rh, atom + noise), as the reference build contracts it); accepted when its cell lies in the grid and holds nothing but VOLUME, and
 *     collision_check passes (RadialHydration.cpp:143-205): over the directions, a 1rh probe
 *     (clamped to the grid) that holds more than VOLUME counts as inside (a third one rejects) and
 *     skips the direction; else a 3rh probe outside the grid scores +2 and ends the direction, one
 *     holding more than VOLUME scores -2 and ends it, a free one +2; then a 5rh probe outside scores
 *     +1, one holding more than VOLUME -1; the candidate passes when score > min_score (0.25) x 3 x 26;
 *   an accepted water marks its cell W_CENTER and the EMPTY cells within r_vdw(O) of x (box
 *     bin +- ceil(r_vdw(O))) W_AREA (SphericalExpander.h:78-115, AtomicOnly: no water VOLUME),
 *     before the next candidate is tried.
 * xyz: n x 3 atom coordinates (double) in the order the generator visits them, ff: their form-factor
 * types; axes: {min x, y, z, bins x, y, z}; noise: n x 26 x 3 (one row per candidate, in candidate
 * order) or NULL for none.  Writes up to cap waters (n x 3) and their candidate indices
 * (atom * 26 + direction) and returns the count.
 */
#define HYD_DIRS 26

static int hyd_directions(double u[HYD_DIRS][3]) {
    const double pi = 3.14159265358979323846;
    const double ang = 2 * pi / 8;
    int n = 0;
    for (double theta = 0; theta <= pi * 0.5; theta += ang)
        for (double phi = 0; phi <= pi * 0.5; phi += ang) {
            double x = cos(phi) * sin(theta), y = sin(phi) * sin(theta), z = cos(theta);
            double s[8][3] = {{x, y, z}, {-x, y, z}, {x, -y, z}, {-x, -y, z},
                              {x, y, -z}, {-x, y, -z}, {x, -y, -z}, {-x, -y, -z}};
            for (int r = 0; r < 8; ++r) {
                double p[3] = {s[r][0], s[r][1], s[r][2]};
                for (int d = 0; d < 3; ++d)
                    if (fabs(p[d]) < 1e-5) p[d] = 0;
                int present = 0;
                for (int k = 0; k < n && !present; ++k) {
                    double dx = u[k][0] - p[0], dy = u[k][1] - p[1], dz = u[k][2] - p[2];
                    present = sqrt(dx * dx + dy * dy + dz * dz) < 1e-5;
                }
                if (!present) {
                    if (n == HYD_DIRS) return -1;
                    u[n][0] = p[0], u[n][1] = p[1], u[n][2] = p[2];
                    ++n;
                }
            }
        }
    return n;
}

void oracle_hydrate_axes(const double* xyz, int64_t n, double* axes) {
    /* Grid(bodies) keeps the running box in a Vector3 deduced from {0, 0, 0}, i.e. of int
     * (Grid.cpp:36): every extent that widens it is truncated toward zero, and diff is an int */
    const double width = 1.0;
    int mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            if (xyz[3 * i + d] < mn[d]) mn[d] = (int)xyz[3 * i + d];
            if (xyz[3 * i + d] > mx[d]) mx[d] = (int)xyz[3 * i + d];
        }
    int diff[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    double scaling = (diff[0] < 50 || diff[1] < 50 || diff[2] < 50) ? 1.0 : 0.25;
    double margin = 2.14 + 1.71 + (-0.35) + 3 * width;
    for (int d = 0; d < 3; ++d) {
        double e = fmax(0.5 * diff[d] * scaling, margin);
        double lo = floor(mn[d] - e - width), hi = ceil(mx[d] + e + width);
        axes[d] = lo;
        axes[3 + d] = (double)(int)((hi - lo) / width);
    }
}

/* The grid's atom state (one byte per cell, the reference's State bits) is kept by the caller between
 * calls, as the reference keeps a molecule's grid across rigid-body steps:
 *   oracle_hgrid_add: Grid::add(body) marks the atoms' cells A_CENTER (Grid.cpp:293-330), and the
 *     volume expansion that hydrate() then runs treats the atoms in order: cells within r_vdw that hold
 *     nothing or VOLUME get A_AREA, cells within (r_vdw, rvol] that hold nothing get VOLUME
 *     (SphericalExpander.h:27-76);
 *   oracle_hgrid_remove: Grid::remove(body) deflates each atom, clearing A_AREA and VOLUME within
 *     max(r_vdw, rvol) whatever else covers those cells, and clears A_CENTER of its cell
 *     (Grid.cpp:372-400, SphericalExpander.h:117-150);
 *   oracle_hgrid_hydrate: the generation on a copy of the state (waters never touch the caller's
 *     state: the reference clears them before each generation, and their removal only clears W_AREA,
 *     SphericalExpander.h:152-186). */
enum { HG_VOLUME = 1, HG_A_CENTER = 4, HG_A_AREA = 8, HG_W_CENTER = 16, HG_W_AREA = 32 };

static void hg_shape(const double* axes, double gmin[3], int bins[3]) {
    for (int d = 0; d < 3; ++d) gmin[d] = axes[d], bins[d] = (int)axes[3 + d];
}

void oracle_hgrid_add(unsigned char* g, const double* axes, const double* xyz, const int32_t* ff, int64_t n) {
    const double width = 1.0, rvol = 2.15;
    double gmin[3];
    int bins[3];
    hg_shape(axes, gmin, bins);
#define CELL(i, j, k) g[((size_t)(i) * bins[1] + (j)) * bins[2] + (k)]
    for (int64_t a = 0; a < n; ++a) {
        int b[3], in = 1;
        for (int d = 0; d < 3; ++d) {
            b[d] = (int)round((xyz[3 * a + d] - gmin[d]) / width);
            in = in && b[d] >= 0 && b[d] < bins[d];
        }
        if (in) CELL(b[0], b[1], b[2]) |= HG_A_CENTER; /* outside: the caller's error (the C ABI rejects it) */
    }
    for (int64_t a = 0; a < n; ++a) {
        const double* p = xyz + 3 * a;
        double rvdw = vdw_of_ff(ff[a]), rvdw2 = rvdw * rvdw, rvol2 = rvol * rvol;
        int br = (int)ceil(fmax(rvdw, rvol) / width);
        int b[3], lo_[3], hi_[3];
        for (int d = 0; d < 3; ++d) {
            b[d] = (int)round((p[d] - gmin[d]) / width);
            lo_[d] = b[d] - br > 0 ? b[d] - br : 0;
            hi_[d] = b[d] + br + 1 < bins[d] ? b[d] + br + 1 : bins[d];
        }
        for (int i = lo_[0]; i < hi_[0]; ++i) {
            double x2 = pow(gmin[0] + i * width - p[0], 2);
            for (int j = lo_[1]; j < hi_[1]; ++j) {
                double x2y2 = x2 + pow(gmin[1] + j * width - p[1], 2);
                for (int k = lo_[2]; k < hi_[2]; ++k) {
                    double dist = x2y2 + pow(gmin[2] + k * width - p[2], 2);
                    unsigned char* c = &CELL(i, j, k);
                    if (dist <= rvdw2) {
                        if (!(*c == 0 || (*c & HG_VOLUME))) continue;
                        *c |= HG_A_AREA;
                    } else if (dist <= rvol2) {
                        if (*c != 0) continue;
                        *c |= HG_VOLUME;
                    }
                }
            }
        }
    }
#undef CELL
}

void oracle_hgrid_remove(unsigned char* g, const double* axes, const double* xyz, const int32_t* ff, int64_t n) {
    const double width = 1.0, rvol = 2.15;
    double gmin[3];
    int bins[3];
    hg_shape(axes, gmin, bins);
#define CELL(i, j, k) g[((size_t)(i) * bins[1] + (j)) * bins[2] + (k)]
    for (int64_t a = 0; a < n; ++a) {
        const double* p = xyz + 3 * a;
        double rmax = fmax(vdw_of_ff(ff[a]), rvol), rmax2 = pow(rmax, 2);
        int br = (int)ceil(rmax / width);
        int b[3], lo_[3], hi_[3];
        for (int d = 0; d < 3; ++d) {
            b[d] = (int)round((p[d] - gmin[d]) / width);
            lo_[d] = b[d] - br > 0 ? b[d] - br : 0;
            hi_[d] = b[d] + br + 1 < bins[d] ? b[d] + br + 1 : bins[d];
        }
        for (int i = lo_[0]; i < hi_[0]; ++i) {
            double x2 = pow(gmin[0] + i * width - p[0], 2);
            for (int j = lo_[1]; j < hi_[1]; ++j) {
                double x2y2 = x2 + pow(gmin[1] + j * width - p[1], 2);
                for (int k = lo_[2]; k < hi_[2]; ++k) {
                    double dist = x2y2 + pow(gmin[2] + k * width - p[2], 2);
                    if (dist <= rmax2) CELL(i, j, k) &= (unsigned char)~(HG_A_AREA | HG_VOLUME);
                }
            }
        }
        if (b[0] >= 0 && b[0] < bins[0] && b[1] >= 0 && b[1] < bins[1] && b[2] >= 0 && b[2] < bins[2])
            CELL(b[0], b[1], b[2]) &= (unsigned char)~HG_A_CENTER;
    }
#undef CELL
}

int64_t oracle_hgrid_hydrate(const unsigned char* state, const double* axes, const double* xyz, const int32_t* ff,
                             int64_t n, const double* noise, double* out, int64_t cap, int64_t* cand_out) {
    const double width = 1.0, rw = 1.71, rh = 1.71 + (-0.35);
    double gmin[3];
    int bins[3];
    hg_shape(axes, gmin, bins);
    double u[HYD_DIRS][3];
    if (hyd_directions(u) != HYD_DIRS) return -2;
    int p1[HYD_DIRS][3], p3[HYD_DIRS][3], p5[HYD_DIRS][3];
    for (int i = 0; i < HYD_DIRS; ++i)
        for (int d = 0; d < 3; ++d) {
            p1[i][d] = (int)(round(rh * u[i][d]) / width);
            p3[i][d] = (int)(round(3 * rh * u[i][d]) / width);
            p5[i][d] = (int)(round(5 * rh * u[i][d]) / width);
        }
    size_t cells = (size_t)bins[0] * bins[1] * bins[2];
    unsigned char* g = malloc(cells ? cells : 1);
    if (!g) return -1;
    memcpy(g, state, cells);
#define CELL(i, j, k) g[((size_t)(i) * bins[1] + (j)) * bins[2] + (k)]
#define FREE_(c) (((c) & ~HG_VOLUME) == 0)
    const double min_points = 0.25 * 3 * HYD_DIRS;
    int64_t m = 0;
    for (int64_t a = 0; a < n; ++a) {
        const double* p = xyz + 3 * a;
        const double reff = vdw_of_ff(ff[a]) + rh;
        for (int r = 0; r < HYD_DIRS; ++r) {
            const double* nz = noise ? noise + 3 * (a * HYD_DIRS + r) : NULL;
            double x[3];
            int b[3], valid = 1;
            for (int d = 0; d < 3; ++d) {
                /* the reference build evaluates atom + u reff + noise as fma(u, reff, atom + noise) */
                x[d] = fma(u[r][d], reff, p[d] + (nz ? nz[d] : 0.0));
                b[d] = (int)round((x[d] - gmin[d]) / width);
                valid = valid && b[d] >= 0 && b[d] < bins[d];
            }
            if (!valid || !FREE_(CELL(b[0], b[1], b[2]))) continue;
            /* collision_check */
            int inside = 0, score = 0, ok = 1;
            for (int i = 0; i < HYD_DIRS && ok; ++i) {
                int q[3];
                for (int d = 0; d < 3; ++d) {
                    q[d] = b[d] + p1[i][d];
                    q[d] = q[d] < 0 ? 0 : (q[d] > bins[d] - 1 ? bins[d] - 1 : q[d]);
                }
                if (!FREE_(CELL(q[0], q[1], q[2]))) {
                    if (2 < ++inside) ok = 0;
                    continue;
                }
                int oob = 0;
                for (int d = 0; d < 3; ++d) {
                    q[d] = b[d] + p3[i][d];
                    oob = oob || q[d] < 0 || q[d] >= bins[d];
                }
                if (oob) {
                    score += 2;
                    continue;
                }
                if (!FREE_(CELL(q[0], q[1], q[2]))) {
                    score -= 2;
                    continue;
                }
                score += 2;
                oob = 0;
                for (int d = 0; d < 3; ++d) {
                    q[d] = b[d] + p5[i][d];
                    oob = oob || q[d] < 0 || q[d] >= bins[d];
                }
                if (oob) {
                    score += 1;
                    continue;
                }
                if (!FREE_(CELL(q[0], q[1], q[2]))) score -= 1;
            }
            if (!ok || score <= min_points) continue;
            /* Grid::add(water, expand = true) */
            CELL(b[0], b[1], b[2]) |= HG_W_CENTER;
            const double rw2 = rw * rw;
            const int br = (int)ceil(rw / width);
            int lo_[3], hi_[3];
            for (int d = 0; d < 3; ++d) {
                lo_[d] = b[d] - br > 0 ? b[d] - br : 0;
                hi_[d] = b[d] + br + 1 < bins[d] ? b[d] + br + 1 : bins[d];
            }
            for (int i = lo_[0]; i < hi_[0]; ++i) {
                double x2 = pow(gmin[0] + i * width - x[0], 2);
                for (int j = lo_[1]; j < hi_[1]; ++j) {
                    double x2y2 = x2 + pow(gmin[1] + j * width - x[1], 2);
                    for (int k = lo_[2]; k < hi_[2]; ++k) {
                        double dist = x2y2 + pow(gmin[2] + k * width - x[2], 2);
                        if (dist <= rw2 && CELL(i, j, k) == 0) CELL(i, j, k) |= HG_W_AREA;
                    }
                }
            }
            if (out && m < cap) {
                out[3 * m] = x[0], out[3 * m + 1] = x[1], out[3 * m + 2] = x[2];
                if (cand_out) cand_out[m] = a * HYD_DIRS + r;
            }
            ++m;
        }
    }
#undef FREE_
#undef CELL
    free(g);
    return m;
}

/* A fresh grid of these atoms (Grid(bodies) with the given axes), then the generation. */
int64_t oracle_hydrate(const double* xyz, const int32_t* ff, int64_t n, const double* axes, const double* noise,
                       double* out, int64_t cap, int64_t* cand_out) {
    size_t cells = (size_t)axes[3] * (size_t)axes[4] * (size_t)axes[5];
    unsigned char* g = calloc(cells ? cells : 1, 1);
    if (!g) return -1;
    oracle_hgrid_add(g, axes, xyz, ff, n);
    int64_t m = oracle_hgrid_hydrate(g, axes, xyz, ff, n, noise, out, cap, cand_out);
    free(g);
    return m;
}
