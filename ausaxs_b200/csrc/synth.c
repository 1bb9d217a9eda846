/*
 * Seeded synthetic structures for the benchmark workloads and the tests (no public dataset is
 * used): protein-like globules, hydration shells and grid excluded-volume dummies.
 *
 * globule : a self-avoiding random walk of 1.5 A steps confined to a sphere (radius chosen for the
 *           requested radius of gyration, R = Rg / sqrt(3/5)) or to a spherical-shell sector,
 *           minimum separation 1.3 A between walk atoms; element C/N/O/S drawn per atom.
 * waters  : points drawn around random atoms, kept when their distance to the nearest atom's
 *           van der Waals surface lies in [shell_min, shell_max] (and, optionally, they keep a
 *           minimum separation from accepted waters).
 * exv grid: one dummy at the centre of every grid cell whose centre lies inside an atom's van der
 *           Waals sphere (the occupied molecular volume).
 * Build: gcc -O2 -fPIC -shared (see ausaxs_b200/build.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t s;
} rng_t;

static uint64_t rng_next(rng_t* r) { /* splitmix64 */
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_u(rng_t* r) { return (rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* ---- uniform cell list over a bounding box ---------------------------------------------- */
typedef struct {
    double lo[3], cell;
    int dim[3];
    int* head;  /* per cell: first point index or -1 */
    int* next;  /* per point */
    int cap;
} grid_t;

static int grid_init(grid_t* g, const double* lo, const double* hi, double cell, int cap) {
    g->cell = cell;
    long long n = 1;
    for (int k = 0; k < 3; ++k) {
        g->lo[k] = lo[k];
        g->dim[k] = (int)ceil((hi[k] - lo[k]) / cell) + 1;
        n *= g->dim[k];
    }
    if (n > 400000000LL) return -1;
    g->head = malloc(sizeof(int) * (size_t)n);
    g->next = malloc(sizeof(int) * (size_t)cap);
    if (!g->head || !g->next) return -1;
    memset(g->head, 0xff, sizeof(int) * (size_t)n);
    g->cap = cap;
    return 0;
}
static void grid_free(grid_t* g) {
    free(g->head);
    free(g->next);
}
static int grid_cell(const grid_t* g, const double* p, int* c) {
    for (int k = 0; k < 3; ++k) {
        c[k] = (int)floor((p[k] - g->lo[k]) / g->cell);
        if (c[k] < 0 || c[k] >= g->dim[k]) return -1;
    }
    return (c[2] * g->dim[1] + c[1]) * g->dim[0] + c[0];
}
static void grid_add(grid_t* g, const double* pts, int i) {
    int c[3];
    int id = grid_cell(g, pts + 3 * i, c);
    if (id < 0) return;
    g->next[i] = g->head[id];
    g->head[id] = i;
}
/* smallest (|p - x_i| - rad_i) over points within reach cells (rad may be NULL: 0); returns early
 * once it is below stop_below (the callers only need to know that) */
static double grid_min_gap(const grid_t* g, const double* pts, const double* rad, const double* p, int reach,
                           double stop_below) {
    int c[3];
    for (int k = 0; k < 3; ++k) c[k] = (int)floor((p[k] - g->lo[k]) / g->cell);
    double best = 1e30;
    for (int dz = -reach; dz <= reach; ++dz)
        for (int dy = -reach; dy <= reach; ++dy)
            for (int dx = -reach; dx <= reach; ++dx) {
                int x = c[0] + dx, y = c[1] + dy, z = c[2] + dz;
                if (x < 0 || y < 0 || z < 0 || x >= g->dim[0] || y >= g->dim[1] || z >= g->dim[2]) continue;
                for (int i = g->head[(z * g->dim[1] + y) * g->dim[0] + x]; i >= 0; i = g->next[i]) {
                    double ex = p[0] - pts[3 * i], ey = p[1] - pts[3 * i + 1], ez = p[2] - pts[3 * i + 2];
                    double d = sqrt(ex * ex + ey * ey + ez * ez) - (rad ? rad[i] : 0.0);
                    if (d < best) {
                        best = d;
                        if (best < stop_below) return best;
                    }
                }
            }
    return best;
}

/* element -> (form_factor_t, vdW radius): C, N, O, S */
static const int FF_OF[4] = {3, 7, 11, 12};
static const double VDW_OF[4] = {1.70, 1.55, 1.52, 1.80};

/*
 * Random-walk globule.  Region: r_in <= |x| <= r_out, and (when cone_cos > -1) inside the cone of
 * half-angle acos(cone_cos) around +z.  frac: cumulative C/N/O/S fractions.  Writes xyz [n][3] and
 * ff [n]; returns the number of atoms placed (n unless the region is too tight).
 */
int synth_globule(uint64_t seed, int n, double r_in, double r_out, double cone_cos, const double* frac, double* xyz,
                  int32_t* ff) {
    rng_t r = {seed * 0x2545F4914F6CDD1Dull + 1};
    const double step = 1.5, min_sep = 1.3;
    double lo[3] = {-r_out - 2, -r_out - 2, -r_out - 2}, hi[3] = {r_out + 2, r_out + 2, r_out + 2};
    grid_t g;
    if (grid_init(&g, lo, hi, 1.5, n) != 0) return -1;
    /* start point inside the region */
    double p[3];
    for (int tries = 0;; ++tries) {
        for (int k = 0; k < 3; ++k) p[k] = (2 * rng_u(&r) - 1) * r_out;
        double rr = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        if (rr >= r_in && rr <= r_out && (cone_cos <= -1 || (rr > 0 && p[2] / rr >= cone_cos))) break;
        if (tries > 1000000) {
            grid_free(&g);
            return 0;
        }
    }
    int placed = 0;
    memcpy(xyz, p, sizeof(p));
    grid_add(&g, xyz, 0);
    placed = 1;
    int cur = 0;
    int stuck = 0;
    while (placed < n) {
        int ok = 0;
        for (int t = 0; t < 64 && !ok; ++t) {
            double u = 2 * rng_u(&r) - 1, phi = 2 * M_PI * rng_u(&r), s = sqrt(1 - u * u);
            double q[3] = {xyz[3 * cur] + step * s * cos(phi), xyz[3 * cur + 1] + step * s * sin(phi), xyz[3 * cur + 2] + step * u};
            double rr = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
            if (rr < r_in || rr > r_out) continue;
            if (cone_cos > -1 && (rr == 0 || q[2] / rr < cone_cos)) continue;
            if (grid_min_gap(&g, xyz, NULL, q, 1, min_sep) < min_sep) continue;
            memcpy(xyz + 3 * placed, q, sizeof(q));
            grid_add(&g, xyz, placed);
            cur = placed;
            ++placed;
            ok = 1;
        }
        if (!ok) {
            cur = (int)(rng_u(&r) * placed); /* branch from an earlier atom */
            if (++stuck > 200 * n) break;
        }
    }
    for (int i = 0; i < placed; ++i) {
        double u = rng_u(&r);
        int e = 3;
        for (int k = 0; k < 4; ++k)
            if (u < frac[k]) {
                e = k;
                break;
            }
        ff[i] = FF_OF[e];
    }
    grid_free(&g);
    return placed;
}

static double vdw_of_ff(int f) {
    for (int k = 0; k < 4; ++k)
        if (FF_OF[k] == f) return VDW_OF[k];
    return 1.7;
}

/* Hydration waters in a [shell_min, shell_max] band outside the atoms' vdW surface. */
int synth_waters(uint64_t seed, const double* xyz, const int32_t* ff, int n, int n_waters, double shell_min,
                 double shell_max, double min_water_sep, double* out) {
    if (n <= 0 || n_waters <= 0) return 0;
    rng_t r = {seed * 0x9E3779B97F4A7C15ull + 7};
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            if (xyz[3 * i + k] < lo[k]) lo[k] = xyz[3 * i + k];
            if (xyz[3 * i + k] > hi[k]) hi[k] = xyz[3 * i + k];
        }
    double pad = shell_max + 2.5;
    for (int k = 0; k < 3; ++k) lo[k] -= pad, hi[k] += pad;
    double* rad = malloc(sizeof(double) * n);
    for (int i = 0; i < n; ++i) rad[i] = vdw_of_ff(ff[i]);
    grid_t g, gw;
    double cell = shell_max + 2.0;
    if (grid_init(&g, lo, hi, cell, n) != 0 || grid_init(&gw, lo, hi, 2.5, n_waters) != 0) {
        free(rad);
        return -1;
    }
    for (int i = 0; i < n; ++i) grid_add(&g, xyz, i);
    int placed = 0;
    long long tries = 0, max_tries = (long long)n_waters * 2000LL;
    while (placed < n_waters && tries < max_tries) {
        ++tries;
        /* sample near a random atom to keep acceptance high */
        int a = (int)(rng_u(&r) * n);
        double u = 2 * rng_u(&r) - 1, phi = 2 * M_PI * rng_u(&r), s = sqrt(1 - u * u);
        double dist = rad[a] + shell_min + (shell_max - shell_min) * rng_u(&r);
        double p[3] = {xyz[3 * a] + dist * s * cos(phi), xyz[3 * a + 1] + dist * s * sin(phi), xyz[3 * a + 2] + dist * u};
        double gap = grid_min_gap(&g, xyz, rad, p, 1, shell_min);
        if (gap < shell_min || gap > shell_max) continue;
        if (min_water_sep > 0 && placed && grid_min_gap(&gw, out, NULL, p, 1, min_water_sep) < min_water_sep) continue;
        memcpy(out + 3 * placed, p, sizeof(p));
        grid_add(&gw, out, placed);
        ++placed;
    }
    grid_free(&g);
    grid_free(&gw);
    free(rad);
    return placed;
}

/* Excluded-volume dummies: centres of width-sized cells inside any atom's vdW sphere.
 * With out == NULL only counts. */
int synth_exv_grid(const double* xyz, const int32_t* ff, int n, double width, double* out, int cap) {
    if (n <= 0) return 0;
    double lo[3] = {1e30, 1e30, 1e30}, hi[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            if (xyz[3 * i + k] < lo[k]) lo[k] = xyz[3 * i + k];
            if (xyz[3 * i + k] > hi[k]) hi[k] = xyz[3 * i + k];
        }
    int dim[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = floor((lo[k] - 2.0) / width) * width;
        dim[k] = (int)ceil((hi[k] + 2.0 - lo[k]) / width) + 1;
    }
    size_t cells = (size_t)dim[0] * dim[1] * dim[2];
    unsigned char* occ = calloc(cells, 1);
    if (!occ) return -1;
    for (int i = 0; i < n; ++i) {
        double rv = vdw_of_ff(ff[i]), r2 = rv * rv;
        int c0[3], c1[3];
        for (int k = 0; k < 3; ++k) {
            c0[k] = (int)floor((xyz[3 * i + k] - rv - lo[k]) / width);
            c1[k] = (int)ceil((xyz[3 * i + k] + rv - lo[k]) / width);
            if (c0[k] < 0) c0[k] = 0;
            if (c1[k] >= dim[k]) c1[k] = dim[k] - 1;
        }
        for (int z = c0[2]; z <= c1[2]; ++z)
            for (int y = c0[1]; y <= c1[1]; ++y)
                for (int x = c0[0]; x <= c1[0]; ++x) {
                    double cx = lo[0] + (x + 0.5) * width - xyz[3 * i];
                    double cy = lo[1] + (y + 0.5) * width - xyz[3 * i + 1];
                    double cz = lo[2] + (z + 0.5) * width - xyz[3 * i + 2];
                    if (cx * cx + cy * cy + cz * cz <= r2) occ[((size_t)z * dim[1] + y) * dim[0] + x] = 1;
                }
    }
    int m = 0;
    for (int z = 0; z < dim[2]; ++z)
        for (int y = 0; y < dim[1]; ++y)
            for (int x = 0; x < dim[0]; ++x)
                if (occ[((size_t)z * dim[1] + y) * dim[0] + x]) {
                    if (out && m < cap) {
                        out[3 * m] = lo[0] + (x + 0.5) * width;
                        out[3 * m + 1] = lo[1] + (y + 0.5) * width;
                        out[3 * m + 2] = lo[2] + (z + 0.5) * width;
                    }
                    ++m;
                }
    free(occ);
    return m;
}
