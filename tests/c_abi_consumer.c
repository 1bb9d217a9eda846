/*
 * A plain C caller of the C ABI (include/ausaxs_b200.h), the way a reference-side binding would use it:
 * the reference's SimpleCube known-answer structure (tests/feature/hist/hist_test_helper.h:87-162 in
 * the reference: 8 carbon atoms on the corners of a 2 A cube plus one in its centre, 8 waters on the
 * corners), HistogramManagerMTFFAvg's calculate_all() and debye_transform(), the grid excluded volume
 * of the cube (149 dummies of 1 A^3 in the reference's RawGridExv), a SimpleCalculator self job with
 * a scaling factor, a noise-free SmartFitter fit of the water scaling, and one error path.
 * Exit status 0 and "ok" when every check holds.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ausaxs_b200.h"

#define NB 8000

static void put(float* rec, double x, double y, double z, int32_t ff) {
    rec[0] = (float)x;
    rec[1] = (float)y;
    rec[2] = (float)z;
    memcpy(&rec[3], &ff, 4);
}

int main(void) {
    float atoms[9][4], waters[8][4];
    int k = 0;
    for (int i = -1; i <= 1; i += 2)
        for (int j = -1; j <= 1; j += 2)
            for (int l = -1; l <= 1; l += 2, ++k) {
                put(atoms[k], i, j, l, 3); /* form_factor_t::C */
                put(waters[k], i, j, l, 1); /* form_factor_t::WATER */
            }
    put(atoms[8], 0, 0, 0, 3);

    ausaxs_gpu_ctx* ctx = NULL;
    if (ausaxs_gpu_ctx_create(0, &ctx) != AUSAXS_OK) {
        fprintf(stderr, "ctx: %s\n", ausaxs_gpu_last_error());
        return 2;
    }
    ausaxs_hist_config cfg = {AUSAXS_MANAGER_FFAVG, 1, 0.25, NB, 100.0 * 0.334 / 9};
    double* aa = calloc((size_t)15 * 15 * NB, sizeof(double));
    double* aw = calloc((size_t)15 * NB, sizeof(double));
    double* ww = calloc(NB, sizeof(double));
    double* tot = calloc(NB, sizeof(double));
    double* d = calloc(NB, sizeof(double));
    ausaxs_hist_result r = {0, 0, 0, aa, aw, ww, tot, d, NULL, NULL};
    if (ausaxs_gpu_histogram(ctx, &cfg, &atoms[0][0], 9, &waters[0][0], 8, NULL, 0, &r) != AUSAXS_OK) {
        fprintf(stderr, "histogram: %s\n", ausaxs_gpu_last_error());
        return 3;
    }
    /* carbon-carbon counts (factor 2, self terms in bin 0): centre-corner sqrt(3) -> bin 7 (8 pairs),
     * edges 2 -> bin 8 (12), face diagonals 2 sqrt(2) -> bin 11 (12), space diagonals 2 sqrt(3) -> bin 14 (4) */
    const int mb = r.max_bin;
    const double* cc = aa + (size_t)(3 * 15 + 3) * mb;
    const double want[15] = {9, 0, 0, 0, 0, 0, 0, 16, 24, 0, 0, 24, 0, 0, 8};
    int bad = mb != 15;
    for (int b = 0; b < 15 && !bad; ++b) bad |= cc[b] != want[b];
    if (bad) {
        fprintf(stderr, "unexpected carbon-carbon histogram (max_bin %d)\n", mb);
        return 4;
    }
    if (fabs(d[8] - 2.0) > 1e-5 || fabs(d[7] - sqrt(3.0)) > 1e-5) {
        fprintf(stderr, "unexpected distance axis %.9f %.9f\n", d[7], d[8]);
        return 5;
    }
    const double q[3] = {0.01, 0.1, 0.5};
    double I[3];
    ausaxs_debye_params p = {1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1, 1e-5};
    if (ausaxs_gpu_debye(ctx, &cfg, &r, q, 3, &p, I, NULL) != AUSAXS_OK) {
        fprintf(stderr, "debye: %s\n", ausaxs_gpu_last_error());
        return 6;
    }
    for (int i = 0; i < 3; ++i)
        if (!isfinite(I[i])) return 7;
    /* grid excluded volume of the cube (the reference's RawGridExv gives 149 dummies, 149 A^3) */
    int64_t n_exv = 0;
    double vol = 0;
    if (ausaxs_gpu_grid_exv(ctx, &atoms[0][0], 9, &waters[0][0], 8, 1, NULL, 0, &n_exv, &vol) != AUSAXS_OK ||
        n_exv != 149 || vol != 149.0) {
        fprintf(stderr, "grid exv: %lld dummies, %.1f A^3 (%s)\n", (long long)n_exv, vol, ausaxs_gpu_last_error());
        return 9;
    }
    /* SimpleCalculator: the cube's atoms with weight 1, scaling 3: factor 6 per pair, 3 * 9 on the diagonal */
    float unit[9][4];
    for (int i = 0; i < 9; ++i) {
        memcpy(unit[i], atoms[i], 3 * sizeof(float));
        unit[i][3] = 1.0f;
    }
    ausaxs_gpu_calculator* calc = NULL;
    int32_t idx = -1, ns = 0, nc = 0;
    double* cv = calloc(NB, sizeof(double));
    double* cn = calloc(NB, sizeof(double));
    if (ausaxs_gpu_calculator_create(ctx, 0.25, NB, &calc) != AUSAXS_OK ||
        ausaxs_gpu_calculator_enqueue_self(calc, &unit[0][0], 9, 3, -1, &idx) != AUSAXS_OK || idx != 0 ||
        ausaxs_gpu_calculator_run(calc, &ns, &nc) != AUSAXS_OK || ns != 1 || nc != 0 ||
        ausaxs_gpu_calculator_result(calc, 0, 0, cv, cn, NULL) != AUSAXS_OK) {
        fprintf(stderr, "calculator: %s\n", ausaxs_gpu_last_error());
        return 10;
    }
    if (cv[0] != 27 || cn[0] != 27 || cv[7] != 48 || cv[8] != 72 || cv[11] != 72 || cv[14] != 24) {
        fprintf(stderr, "calculator values %g %g %g %g %g\n", cv[0], cv[7], cv[8], cv[11], cv[14]);
        return 11;
    }
    ausaxs_gpu_calculator_destroy(calc);
    /* SmartFitter: data = 3 * I(cw = 2) + 5 on 20 q values; the water scaling comes back as 2 */
    double fq[20], fI[20], fs[20];
    for (int i = 0; i < 20; ++i) fq[i] = 0.01 + 0.02 * i;
    ausaxs_debye_params p2 = p;
    p2.cw = 2.0;
    if (ausaxs_gpu_debye(ctx, &cfg, &r, fq, 20, &p2, fI, NULL) != AUSAXS_OK) return 12;
    for (int i = 0; i < 20; ++i) {
        fI[i] = 3 * fI[i] + 5;
        fs[i] = 0.01 * fI[i];
    }
    ausaxs_fit_options opt = {0, 0.0, 0.0, 1e-4};
    ausaxs_fit_result fit;
    if (ausaxs_gpu_fit(ctx, &cfg, &r, fq, fI, fs, 20, &p, &opt, &fit, NULL) != AUSAXS_OK ||
        fabs(fit.value - 2.0) > 1e-4 || fabs(fit.a - 3.0) > 1e-3 || fit.chi2 > 1e-2) {
        fprintf(stderr, "fit: cw %.6f a %.6f chi2 %.3g (%s)\n", fit.value, fit.a, fit.chi2, ausaxs_gpu_last_error());
        return 13;
    }
    /* errors come back as status codes plus text, never as a crash */
    if (ausaxs_gpu_histogram(ctx, &cfg, &atoms[0][0], -1, NULL, 0, NULL, 0, &r) != AUSAXS_ERR_ARGUMENT ||
        strlen(ausaxs_gpu_last_error()) == 0)
        return 8;
    ausaxs_gpu_ctx_destroy(ctx);
    free(aa);
    free(aw);
    free(ww);
    free(tot);
    free(d);
    free(cv);
    free(cn);
    printf("ok I(0.01)=%.6e I(0.1)=%.6e I(0.5)=%.6e\n", I[0], I[1], I[2]);
    return 0;
}
