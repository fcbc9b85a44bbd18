/*
 * FP64 CPU oracle for the tiled fixed-bandwidth Gaussian KDE path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the "port" CPU
 * baseline.  The product never links or calls it.  See oracle.h for the
 * contract of each function and the reference lines it restates.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  FMA
 * contraction is off so the float parts that are reproduced bit for bit
 * (rule of thumb) round exactly as the reference's scalar code does.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Utilities.h:8 — TWO_PI is a float constant in the reference. */
static const double kTwoPiF = (double)6.2831853071795862f;
/* Utilities.h:20 — EPSILONDENSITY is a float constant. */
static const double kEpsDensity = (double)0.00000000000001f;
/* Utilities.h:27 — CUT_OFF_FACTOR. */
static const double kCut = 9.0;

static int g_threads = 0;

void orc_set_threads(int n) { g_threads = n; }

int orc_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

float orc_cell_x(const orc_grid* g, int64_t col) {
    /* COL_TO_XCOORD(COL, XLL, CS) = XLL + (COL + 0.5) * CS, Utilities.h:14 */
    return (float)((double)g->xll + ((double)col + 0.5) * (double)g->cs);
}

float orc_cell_y(const orc_grid* g, int64_t row) {
    /* ROW_TO_YCOORD(ROW, NROWS, YLL, CS) = YLL + (NROWS - 0.5 - ROW) * CS, Utilities.h:13 */
    return (float)((double)g->yll + ((double)g->nrows - 0.5 - (double)row) * (double)g->cs);
}

double orc_h2(float h) {
    float hh = h * h; /* float product, kde_cuda_kdtr_tiled.cu:716 `hp * hp` */
    return (double)hh;
}

/* Exact squared distance of two float positions. */
static inline double d2_exact(float x0, float y0, float x1, float y1) {
    double dx = (double)x1 - (double)x0;
    double dy = (double)y1 - (double)y0;
    return dx * dx + dy * dy;
}

/* The reference's Distance2 (kde_cuda_kdtr_tiled.cu:50-55): float
 * differences widened to double.  Used only where the reference's scalar
 * result is reproduced bit for bit (rule of thumb). */
static inline double d2_ref(float x0, float y0, float x1, float y1) {
    double dx = (double)(x1 - x0);
    double dy = (double)(y1 - y0);
    return dx * dx + dy * dy;
}

/* Gaussian kernel value, kde_cuda_kdtr_tiled.cu:71-76, without the cutoff
 * test (callers test d2 < 9 h2 exactly as the reference does). */
static inline double kern(double h2, double d2) {
    return exp(d2 / (-2.0 * h2)) / (h2 * kTwoPiF);
}

float orc_rule_of_thumb(int64_t n, const float* x, const float* y, const float* w) {
    /* MeanCenter, :1563-1579: float accumulators. */
    float sum_x = 0.0f, sum_y = 0.0f, sum_w = 0.0f;
    for (int64_t p = 0; p < n; p++) {
        float w_p = w ? w[p] : 1.0f;
        sum_w += w_p;
        sum_x += w_p * x[p];
        sum_y += w_p * y[p];
    }
    float mean_x = sum_x / sum_w;
    float mean_y = sum_y / sum_w;
    /* StandardDistance2, :1582-1595: double accumulators. */
    double sum2 = 0.0, sumw = 0.0;
    for (int64_t p = 0; p < n; p++) {
        float w_p = w ? w[p] : 1.0f;
        sumw += w_p;
        sum2 += w_p * d2_ref(mean_x, mean_y, x[p], y[p]);
    }
    double d2 = sum2 / sumw;
    /* BandWidth2, :64-68, then sqrtf at :481. */
    unsigned int three_n = 3u * (unsigned int)n;
    double bw2 = (double)sqrtf(2.0f / (float)three_n) * d2;
    return sqrtf((float)bw2);
}

void orc_mark_boundary(const orc_grid* g, const float* mask, uint8_t* out) {
    const int64_t nc = g->ncols, nr = g->nrows;
    const float nd = g->nodata;
#pragma omp parallel for num_threads(orc_get_threads()) schedule(static)
    for (int64_t r = 0; r < nr; r++) {
        for (int64_t c = 0; c < nc; c++) {
            int64_t i = r * nc + c;
            uint8_t b = 0;
            if (mask[i] != nd) {
                if (r == 0 || r == nr - 1 || c == 0 || c == nc - 1) {
                    b = 1;
                } else {
                    for (int dr = -1; dr <= 1 && !b; dr++)
                        for (int dc = -1; dc <= 1; dc++) {
                            if (dr == 0 && dc == 0) continue;
                            if (mask[(r + dr) * nc + (c + dc)] == nd) { b = 1; break; }
                        }
                }
            }
            out[i] = b;
        }
    }
}

void orc_dist2_boundary(int64_t n, const float* x, const float* y,
                        const orc_grid* g, const uint8_t* boundary, double* out) {
    /* Compact the boundary-cell centres once (the reference's serialized
     * raster, :3985-3986), then brute force in double as :4092-4133. */
    const int64_t nc = g->ncols, nr = g->nrows;
    int64_t nb = 0;
    for (int64_t i = 0; i < nc * nr; i++) nb += boundary[i] ? 1 : 0;
    float* bx = (float*)malloc(sizeof(float) * (size_t)(nb > 0 ? nb : 1));
    float* by = (float*)malloc(sizeof(float) * (size_t)(nb > 0 ? nb : 1));
    int64_t k = 0;
    for (int64_t r = 0; r < nr; r++)
        for (int64_t c = 0; c < nc; c++)
            if (boundary[r * nc + c]) {
                bx[k] = orc_cell_x(g, c);
                by[k] = orc_cell_y(g, r);
                k++;
            }
#pragma omp parallel for num_threads(orc_get_threads()) schedule(dynamic, 64)
    for (int64_t p = 0; p < n; p++) {
        double best = DBL_MAX;
        for (int64_t j = 0; j < nb; j++) {
            double d2 = d2_exact(x[p], y[p], bx[j], by[j]);
            if (d2 < best) best = d2;
        }
        out[p] = best;
    }
    free(bx);
    free(by);
}

static const double* g_sort_keys;

static int cmp_order(const void* a, const void* b) {
    int64_t ia = *(const int64_t*)a, ib = *(const int64_t*)b;
    double da = g_sort_keys[ia], db = g_sort_keys[ib];
    if (da < db) return -1;
    if (da > db) return 1;
    return ia < ib ? -1 : (ia > ib ? 1 : 0);
}

void orc_sort_order(int64_t n, const double* dist2, int64_t* order) {
    for (int64_t i = 0; i < n; i++) order[i] = i;
    g_sort_keys = dist2;
    qsort(order, (size_t)n, sizeof(int64_t), cmp_order);
}

/* YCOORD_TO_ROW / XCOORD_TO_COL, Utilities.h:16-17 (truncating casts). */
static inline int64_t y_to_row(double yv, const orc_grid* g) {
    return g->nrows - 1 - (int64_t)(int)((yv - (double)g->yll) / (double)g->cs);
}
static inline int64_t x_to_col(double xv, const orc_grid* g) {
    return (int64_t)(int)((xv - (double)g->xll) / (double)g->cs);
}

void orc_edge_weights(int64_t n, const float* x, const float* y,
                      const float* hs, float h, const double* dist2,
                      const orc_grid* g, const float* mask,
                      double* out, int64_t* evals) {
    const double cell_area = (double)(g->cs * g->cs); /* float product, :2698 */
    int64_t total = 0;
#pragma omp parallel for num_threads(orc_get_threads()) schedule(dynamic, 16) reduction(+ : total)
    for (int64_t p = 0; p < n; p++) {
        const float hp = hs ? hs[p] : h;
        const double h2 = orc_h2(hp);
        if (dist2 && dist2[p] >= kCut * h2) { /* short-circuit, :2704-2708 */
            out[p] = 1.0;
            continue;
        }
        const float px = x[p], py = y[p];
        /* NARROW window, :2719-2727 (a superset of the 3h disc). */
        int64_t rl = y_to_row((double)py + 3.0 * hp, g);
        int64_t ru = y_to_row((double)py - 3.0 * hp, g);
        int64_t cl = x_to_col((double)px - 3.0 * hp, g);
        int64_t cu = x_to_col((double)px + 3.0 * hp, g);
        if (rl < 0) rl = 0;
        if (ru > g->nrows - 1) ru = g->nrows - 1;
        if (cl < 0) cl = 0;
        if (cu > g->ncols - 1) cu = g->ncols - 1;
        double acc = 0.0;
        int64_t cnt = 0;
        for (int64_t r = rl; r <= ru; r++) {
            const float cy = orc_cell_y(g, r);
            for (int64_t c = cl; c <= cu; c++) {
                if (mask[r * g->ncols + c] == g->nodata) continue;
                const double d2 = d2_exact(px, py, orc_cell_x(g, c), cy);
                if (d2 < kCut * h2) {
                    acc += kern(h2, d2) * cell_area;
                    cnt++;
                }
            }
        }
        out[p] = 1.0 / acc;
        total += cnt;
    }
    if (evals) *evals = total;
}

/* ---- cell-binned candidate lists (oracle-side acceleration only) ---- */
typedef struct {
    double x0, y0, side;
    int64_t nbx, nby;
    int64_t* start; /* nbx*nby + 1 */
    int64_t* idx;   /* point indices, bin-major, ascending within a bin */
} bins_t;

static void bins_build(bins_t* b, int64_t n, const float* x, const float* y, double side) {
    double xmin = DBL_MAX, ymin = DBL_MAX, xmax = -DBL_MAX, ymax = -DBL_MAX;
    for (int64_t i = 0; i < n; i++) {
        if (x[i] < xmin) xmin = x[i];
        if (x[i] > xmax) xmax = x[i];
        if (y[i] < ymin) ymin = y[i];
        if (y[i] > ymax) ymax = y[i];
    }
    if (n == 0) { xmin = ymin = 0.0; xmax = ymax = 1.0; }
    if (!(side > 0.0)) side = 1.0;
    b->x0 = xmin;
    b->y0 = ymin;
    b->side = side;
    b->nbx = (int64_t)floor((xmax - xmin) / side) + 1;
    b->nby = (int64_t)floor((ymax - ymin) / side) + 1;
    /* Bound the bin count for degenerate inputs (huge extent, tiny h). */
    while (b->nbx * b->nby > (int64_t)1 << 24) {
        b->side *= 2.0;
        b->nbx = (int64_t)floor((xmax - xmin) / b->side) + 1;
        b->nby = (int64_t)floor((ymax - ymin) / b->side) + 1;
    }
    const int64_t nb = b->nbx * b->nby;
    b->start = (int64_t*)calloc((size_t)nb + 1, sizeof(int64_t));
    b->idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    int64_t* bin_of = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) {
        int64_t bx = (int64_t)floor(((double)x[i] - b->x0) / b->side);
        int64_t by = (int64_t)floor(((double)y[i] - b->y0) / b->side);
        if (bx < 0) bx = 0;
        if (bx >= b->nbx) bx = b->nbx - 1;
        if (by < 0) by = 0;
        if (by >= b->nby) by = b->nby - 1;
        bin_of[i] = by * b->nbx + bx;
        b->start[bin_of[i] + 1]++;
    }
    for (int64_t k = 0; k < nb; k++) b->start[k + 1] += b->start[k];
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)nb);
    memcpy(cur, b->start, sizeof(int64_t) * (size_t)nb);
    for (int64_t i = 0; i < n; i++) b->idx[cur[bin_of[i]]++] = i;
    free(cur);
    free(bin_of);
}

static void bins_free(bins_t* b) {
    free(b->start);
    free(b->idx);
}

/* Sources sorted by bin with their data stored contiguously, so that a
 * query streams through memory instead of gathering by index.  Bins of side
 * about h_max; a query at (qx, qy) with reach R visits, per bin row within R,
 * only the bins that the disc of radius R reaches in that row.  Points are
 * binned with floor((v - o) / side) in double, which is monotone in v, so the
 * visited bins hold every source within R of the query (the candidate set is
 * a superset of the in-cutoff pairs; the cutoff test itself is unchanged). */
typedef struct {
    bins_t b;
    float* x;      /* bin-major copies of the sources */
    float* y;
    double* w;     /* (double) weight, or 1 */
    double* e;     /* edge weight, or 1 */
    double* h2;    /* orc_h2 of the source's bandwidth */
    int64_t* id;   /* original index */
} sbins_t;

static void sbins_build(sbins_t* s, int64_t n, const float* x, const float* y, const float* w,
                        const double* ew, const float* hs, float h, double side) {
    bins_build(&s->b, n, x, y, side);
    const size_t nn = (size_t)(n > 0 ? n : 1);
    s->x = (float*)malloc(sizeof(float) * nn);
    s->y = (float*)malloc(sizeof(float) * nn);
    s->w = (double*)malloc(sizeof(double) * nn);
    s->e = (double*)malloc(sizeof(double) * nn);
    s->h2 = (double*)malloc(sizeof(double) * nn);
    s->id = s->b.idx;
    for (int64_t t = 0; t < n; t++) {
        const int64_t i = s->b.idx[t];
        s->x[t] = x[i];
        s->y[t] = y[i];
        s->w[t] = (double)(w ? w[i] : 1.0f);
        s->e[t] = ew ? ew[i] : 1.0;
        s->h2[t] = orc_h2(hs ? hs[i] : h);
    }
}

static void sbins_free(sbins_t* s) {
    free(s->x);
    free(s->y);
    free(s->w);
    free(s->e);
    free(s->h2);
    bins_free(&s->b);
}

/* Bin rows [*by0, *by1] within reach R of qy. */
static inline void sbins_rows(const sbins_t* s, double qy, double R, int64_t* by0, int64_t* by1) {
    const bins_t* b = &s->b;
    int64_t l = (int64_t)floor((qy - R - b->y0) / b->side);
    int64_t u = (int64_t)floor((qy + R - b->y0) / b->side);
    *by0 = l < 0 ? 0 : l;
    *by1 = u > b->nby - 1 ? b->nby - 1 : u;
}

/* Candidate range [*t0, *t1) of bin row by for a query at (qx, qy), reach R:
 * the row's bins that intersect the disc's chord at the row's nearest y. */
static inline void sbins_row_range(const sbins_t* s, int64_t by, double qx, double qy, double R,
                                   int64_t* t0, int64_t* t1) {
    const bins_t* b = &s->b;
    const double rlo = b->y0 + (double)by * b->side, rhi = rlo + b->side;
    double dy = qy < rlo ? rlo - qy : (qy > rhi ? qy - rhi : 0.0);
    dy *= 1.0 - 1e-9;
    const double rr = R * R - dy * dy;
    *t0 = *t1 = 0;
    if (rr < 0.0) return;
    const double hw = sqrt(rr) * (1.0 + 1e-9);
    int64_t l = (int64_t)floor((qx - hw - b->x0) / b->side);
    int64_t u = (int64_t)floor((qx + hw - b->x0) / b->side);
    if (l < 0) l = 0;
    if (u > b->nbx - 1) u = b->nbx - 1;
    if (l > u) return;
    *t0 = b->start[by * b->nbx + l];
    *t1 = b->start[by * b->nbx + u + 1];
}

void orc_density(int64_t n, const float* x, const float* y, const float* w,
                 const double* ew, const float* hs, float h,
                 const orc_grid* g, const float* mask,
                 int64_t r0, int64_t c0, int64_t nr, int64_t nc,
                 double* out, int64_t* evals, int brute) {
    float hmax = h;
    if (hs) {
        hmax = 0.0f;
        for (int64_t i = 0; i < n; i++)
            if (hs[i] > hmax) hmax = hs[i];
    }
    sbins_t sb;
    memset(&sb, 0, sizeof(sb));
    if (!brute) sbins_build(&sb, n, x, y, w, ew, hs, h, (double)hmax);
    const double reach = 3.0 * (double)hmax * (1.0 + 1e-6); /* 9h^2 uses the float square */
    int64_t total = 0;
#pragma omp parallel for num_threads(orc_get_threads()) schedule(dynamic, 1) reduction(+ : total)
    for (int64_t rr = 0; rr < nr; rr++) {
        const int64_t r = r0 + rr;
        const float cy = orc_cell_y(g, r);
        for (int64_t cc = 0; cc < nc; cc++) {
            const int64_t c = c0 + cc;
            double* o = &out[rr * nc + cc];
            if (mask && mask[r * g->ncols + c] == g->nodata) {
                *o = (double)g->nodata;
                continue;
            }
            const float cx = orc_cell_x(g, c);
            double den = 0.0;
            int64_t cnt = 0;
            if (brute) {
                for (int64_t p = 0; p < n; p++) {
                    const double h2 = orc_h2(hs ? hs[p] : h);
                    const double d2 = d2_exact(x[p], y[p], cx, cy);
                    if (d2 < kCut * h2) {
                        den += kern(h2, d2) * (double)(w ? w[p] : 1.0f) * (ew ? ew[p] : 1.0);
                        cnt++;
                    }
                }
            } else {
                int64_t by0, by1;
                sbins_rows(&sb, (double)cy, reach, &by0, &by1);
                for (int64_t by = by0; by <= by1; by++) {
                    int64_t t0, t1;
                    sbins_row_range(&sb, by, (double)cx, (double)cy, reach, &t0, &t1);
                    for (int64_t t = t0; t < t1; t++) {
                        const double h2 = sb.h2[t];
                        const double d2 = d2_exact(sb.x[t], sb.y[t], cx, cy);
                        if (d2 < kCut * h2) {
                            den += kern(h2, d2) * sb.w[t] * sb.e[t];
                            cnt++;
                        }
                    }
                }
            }
            *o = den;
            total += cnt;
        }
    }
    if (!brute) sbins_free(&sb);
    if (evals) *evals = total;
}

double orc_loo_loglik(int64_t n, const float* x, const float* y, const float* w,
                      const double* ew, float h, double* out_loo, int64_t* evals) {
    const double h2 = orc_h2(h);
    sbins_t sb;
    sbins_build(&sb, n, x, y, w, ew, NULL, h, (double)h);
    const double reach = 3.0 * (double)h * (1.0 + 1e-6); /* 9h^2 uses the float square */
    double* loo = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    int64_t total = 0;
#pragma omp parallel for num_threads(orc_get_threads()) schedule(dynamic, 64) reduction(+ : total)
    for (int64_t j = 0; j < n; j++) {
        int64_t by0, by1;
        sbins_rows(&sb, (double)y[j], reach, &by0, &by1);
        double den = 0.0;
        int64_t cnt = 0;
        for (int64_t by = by0; by <= by1; by++) {
            int64_t t0, t1;
            sbins_row_range(&sb, by, (double)x[j], (double)y[j], reach, &t0, &t1);
            for (int64_t t = t0; t < t1; t++) {
                if (sb.id[t] == j) continue;
                const double d2 = d2_exact(sb.x[t], sb.y[t], x[j], y[j]);
                if (d2 < kCut * h2) {
                    den += kern(h2, d2) * sb.w[t] * sb.e[t];
                    cnt++;
                }
            }
        }
        loo[j] = den;
        total += cnt;
    }
    /* the log sum in point order (reproducible for any thread count) */
    double logl = 0.0;
    for (int64_t j = 0; j < n; j++) logl += log(loo[j] > kEpsDensity ? loo[j] : kEpsDensity);
    if (out_loo) memcpy(out_loo, loo, sizeof(double) * (size_t)n);
    free(loo);
    sbins_free(&sb);
    if (evals) *evals = total;
    return logl;
}

double orc_loglik_at(int64_t n, const float* x, const float* y, const float* w,
                     const double* dist2, const orc_grid* g, const float* mask,
                     float h, int64_t* evals) {
    double* ew = NULL;
    int64_t e_edge = 0, e_loo = 0;
    if (dist2) {
        ew = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        orc_edge_weights(n, x, y, NULL, h, dist2, g, mask, ew, &e_edge);
    }
    double l = orc_loo_loglik(n, x, y, w, ew, h, NULL, &e_loo);
    free(ew);
    if (evals) *evals = e_edge + e_loo;
    return l;
}

float orc_mle_fixed_bandwidth(int64_t n, const float* x, const float* y, const float* w,
                              const double* dist2, const orc_grid* g, const float* mask,
                              float h0, int* iterations) {
    float hA = h0 / 20;
    float hD = 2 * h0;
    float width = hD - hA;
    float epsilon = width / 100;
    float factor = 1 + sqrtf(5.0f);
    int it = 0;
    while (width > epsilon && it < 30) { /* MAX_NUM_ITERATIONS, Utilities.h:36 */
        float hB = hA + width / factor;
        float hC = hD - width / factor;
        double lB = orc_loglik_at(n, x, y, w, dist2, g, mask, hB, NULL);
        double lC = orc_loglik_at(n, x, y, w, dist2, g, mask, hC, NULL);
        if (lB > lC)
            hD = hC;
        else
            hA = hB;
        width = hD - hA;
        it++;
    }
    if (iterations) *iterations = it;
    return (hA + hD) / 2;
}

/* ---- adaptive bandwidths (h_option 2) ---- */

void orc_point_density(int64_t n, const float* x, const float* y, const float* w,
                       const double* ew, const float* hs, float h, int self,
                       double* out, int64_t* evals) {
    float hmax = h;
    if (hs)
        for (int64_t i = 0; i < n; i++)
            if (hs[i] > hmax) hmax = hs[i];
    sbins_t sb;
    sbins_build(&sb, n, x, y, w, ew, hs, h, (double)hmax);
    const double reach = 3.0 * (double)hmax * (1.0 + 1e-6);
    int64_t total = 0;
#pragma omp parallel for num_threads(orc_get_threads()) schedule(dynamic, 64) reduction(+ : total)
    for (int64_t j = 0; j < n; j++) {
        int64_t by0, by1;
        sbins_rows(&sb, (double)y[j], reach, &by0, &by1);
        double den = 0.0;
        int64_t cnt = 0;
        for (int64_t by = by0; by <= by1; by++) {
            int64_t t0, t1;
            sbins_row_range(&sb, by, (double)x[j], (double)y[j], reach, &t0, &t1);
            for (int64_t t = t0; t < t1; t++) {
                if (sb.id[t] == j && !self) continue;
                const double h2 = sb.h2[t];
                const double d2 = d2_exact(sb.x[t], sb.y[t], x[j], y[j]);
                if (d2 < kCut * h2) {
                    den += kern(h2, d2) * sb.w[t] * sb.e[t];
                    cnt++;
                }
            }
        }
        out[j] = den;
        total += cnt;
    }
    sbins_free(&sb);
    if (evals) *evals = total;
}

void orc_adaptive_bandwidths(int64_t n, const double* den0, float h, float alpha, float* hs) {
    double s = 0.0;
    for (int64_t i = 0; i < n; i++) s += log(den0[i]);
    const double gml = exp(s / (double)n);
    for (int64_t i = 0; i < n; i++) hs[i] = (float)((double)h * pow(den0[i] / gml, (double)alpha));
}

double orc_loglik_adaptive(int64_t n, const float* x, const float* y, const float* w,
                           const double* dist2, const orc_grid* g, const float* mask,
                           float h, float alpha, float* hs_out) {
    const size_t nn = (size_t)(n > 0 ? n : 1);
    double* ew = dist2 ? (double*)malloc(sizeof(double) * nn) : NULL;
    double* den = (double*)malloc(sizeof(double) * nn);
    float* hs = (float*)malloc(sizeof(float) * nn);
    if (dist2) orc_edge_weights(n, x, y, NULL, h, dist2, g, mask, ew, NULL);
    orc_point_density(n, x, y, w, ew, NULL, h, 1, den, NULL);
    orc_adaptive_bandwidths(n, den, h, alpha, hs);
    if (dist2) orc_edge_weights(n, x, y, hs, 0.0f, dist2, g, mask, ew, NULL);
    orc_point_density(n, x, y, w, ew, hs, 0.0f, 0, den, NULL);
    double logl = 0.0;
    for (int64_t j = 0; j < n; j++) logl += log(den[j] > kEpsDensity ? den[j] : kEpsDensity);
    if (hs_out) memcpy(hs_out, hs, sizeof(float) * (size_t)n);
    free(ew);
    free(den);
    free(hs);
    return logl;
}

/* hj_likelihood, kde_cuda_kdtr_tiled.cu:3677-3720: the likelihoods of the
 * centre and its four neighbours, skipping the ones the last move kept.
 * They are kept as floats, the type of the reference's Ls array, so ties and
 * near-ties compare as they do there. */
static void hj_likelihoods(int64_t n, const float* x, const float* y, const float* w, const double* dist2,
                           const orc_grid* g, const float* mask, float h0, float a0, float sh, float sa,
                           int last, float* L) {
    if (last == -1) L[0] = (float)orc_loglik_adaptive(n, x, y, w, dist2, g, mask, h0, a0, NULL);
    if (last != 2) L[1] = (float)orc_loglik_adaptive(n, x, y, w, dist2, g, mask, h0 - sh, a0, NULL);
    if (last != 1) L[2] = (float)orc_loglik_adaptive(n, x, y, w, dist2, g, mask, h0 + sh, a0, NULL);
    if (last != 4) L[3] = (float)orc_loglik_adaptive(n, x, y, w, dist2, g, mask, h0, a0 + sa, NULL);
    if (last != 3) L[4] = (float)orc_loglik_adaptive(n, x, y, w, dist2, g, mask, h0, a0 - sa, NULL);
}

void orc_adaptive_search(int64_t n, const float* x, const float* y, const float* w,
                         const double* dist2, const orc_grid* g, const float* mask,
                         float h0, float* out3, float* hs, int* iterations) {
    float alpha0 = -0.5f;
    float stepH = h0 / 10;
    float stepA = 0.1f;
    float L[5];
    hj_likelihoods(n, x, y, w, dist2, g, mask, h0, alpha0, stepH, stepA, -1, L);
    float Lmax = L[0];
    const float s = stepH / 10;
    const float a = stepA / 10;
    int it = 0;
    while ((stepH > s || stepA > a) && (h0 - stepH > 0) && it <= 30) { /* MAX_NUM_ITERATIONS */
        int dmax = 0;
        for (int i = 0; i < 5; i++)
            if (L[i] > Lmax) {
                Lmax = L[i];
                dmax = i;
            }
        if (dmax == 0) {
            stepH = stepH / 2;
            stepA = stepA / 2;
        } else {
            /* the moves and likelihood bookkeeping of hooke_jeeves (:3750-3778),
             * including its handling of a move to +stepA */
            if (dmax == 1) {
                h0 = h0 - stepH;
                L[2] = L[0];
                L[0] = L[1];
            }
            if (dmax == 2) {
                h0 = h0 + stepH;
                L[1] = L[0];
                L[0] = L[2];
            }
            if (dmax == 3) {
                alpha0 = alpha0 + stepA;
                L[3] = L[0];
                L[0] = L[4];
            }
            if (dmax == 4) {
                alpha0 = alpha0 - stepA;
                L[3] = L[0];
                L[0] = L[4];
            }
        }
        hj_likelihoods(n, x, y, w, dist2, g, mask, h0, alpha0, stepH, stepA, dmax, L);
        it++;
    }
    out3[0] = h0;
    out3[1] = alpha0;
    out3[2] = Lmax;
    if (iterations) *iterations = it;
    /* final bandwidths, main :566-572 */
    const size_t nn = (size_t)(n > 0 ? n : 1);
    double* ew = dist2 ? (double*)malloc(sizeof(double) * nn) : NULL;
    double* den = (double*)malloc(sizeof(double) * nn);
    if (dist2) orc_edge_weights(n, x, y, NULL, h0, dist2, g, mask, ew, NULL);
    orc_point_density(n, x, y, w, ew, NULL, h0, 1, den, NULL);
    orc_adaptive_bandwidths(n, den, h0, alpha0, hs);
    free(ew);
    free(den);
}
