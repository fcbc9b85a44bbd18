/*
 * FP64 CPU oracle for the tiled fixed-bandwidth Gaussian KDE path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, the
 * host driver, the Python package) links, loads or calls this code.  It is
 * the checker that the CUDA path is compared against, and the "port" CPU
 * baseline that bench.py times beside the GPU.
 *
 * Every function is a double-precision restatement of the reference's own
 * sequential (OpenMP CPU) path; each cites the reference lines it follows.
 * Inputs keep the reference's types (float coordinates, weights and
 * bandwidths; float cell-centre coordinates), arithmetic after that is FP64.
 *
 * Parity pin: the restatement is checked against outputs of the reference
 * program itself, built from its own sources by oracle/ref_build.sh and run
 * here (tests/golden/make_golden.py writes the fixtures).
 */
#ifndef MGK_ORACLE_H
#define MGK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Raster geometry, the fields of the reference's AsciiRaster
 * (AsciiRaster.h:9-33) that the path reads.  Row 0 is the top row. */
typedef struct {
    int64_t ncols;
    int64_t nrows;
    float xll;      /* x of the lower-left corner  */
    float yll;      /* y of the lower-left corner  */
    float cs;       /* cell size                   */
    float nodata;   /* NoData value                */
} orc_grid;

/* Cell-centre coordinates, Utilities.h:13-14 (computed in double, stored
 * to float exactly like `cell_x = COL_TO_XCOORD(...)`). */
float orc_cell_x(const orc_grid* g, int64_t col);
float orc_cell_y(const orc_grid* g, int64_t row);

/* Squared bandwidth as the CPU path forms it: a float product widened to
 * double (kde_cuda_kdtr_tiled.cu:2700, :716 `hp * hp`). */
double orc_h2(float h);

/* Rule-of-thumb bandwidth, kde_cuda_kdtr_tiled.cu:64-68, 481, 1563-1595.
 * Follows the reference's own float/double mix exactly (it is a scalar
 * that feeds everything else, so it is reproduced bit for bit). */
float orc_rule_of_thumb(int64_t n, const float* x, const float* y, const float* w);

/* Boundary marking, kde_cuda_kdtr_tiled.cu:3994-4062: a valid cell is a
 * boundary cell if it sits on the raster's outer ring or any of its 8
 * neighbours is NoData.  out[i] = 1 for boundary cells, else 0. */
void orc_mark_boundary(const orc_grid* g, const float* mask, uint8_t* out);

/* Squared distance from each point to the nearest boundary-cell centre,
 * kde_cuda_kdtr_tiled.cu:4092-4133 (CPU branch, double minDist, DBL_MAX
 * when there is no boundary cell). */
void orc_dist2_boundary(int64_t n, const float* x, const float* y,
                        const orc_grid* g, const uint8_t* boundary, double* out);

/* Stable order of points by boundary distance (qsort by distance with the
 * index as tiebreak, kde_cuda_kdtr_tiled.cu:4152-4181). */
void orc_sort_order(int64_t n, const double* dist2, int64_t* order);

/* Exact edge-correction weights, kde_cuda_kdtr_tiled.cu:2694-2807.
 * hs == NULL -> fixed h.  dist2 == NULL -> no short-circuit.
 * Weight = 1 when dist2 >= 9 h^2, else 1 / sum(K * cellArea) over valid
 * mask cells with d^2 < 9 h^2.  evals (optional) receives the number of
 * in-cutoff (point, mask cell) pairs. */
void orc_edge_weights(int64_t n, const float* x, const float* y,
                      const float* hs, float h, const double* dist2,
                      const orc_grid* g, const float* mask,
                      double* out, int64_t* evals);

/* Density on the window [r0, r0+nr) x [c0, c0+nc) of grid g,
 * kde_cuda_kdtr_tiled.cu:707-733 (file mode) and :806-832 (mode 0):
 *   den(c) = sum_p [d^2 < 9 h_p^2] exp(-d^2 / 2h_p^2) / (h_p^2 * TWO_PI) * w_p * e_p
 * for valid cells; NoData cells get the NoData value.  mask == NULL means
 * every cell is valid.  ew == NULL means unit edge weights.  A cell-binned
 * candidate filter (bins of side 3 h_max) replaces the brute-force loop; it
 * sums exactly the same terms.  brute != 0 forces the reference's loop over
 * all points (used by the tests to prove the two equal). */
void orc_density(int64_t n, const float* x, const float* y, const float* w,
                 const double* ew, const float* hs, float h,
                 const orc_grid* g, const float* mask,
                 int64_t r0, int64_t c0, int64_t nr, int64_t nc,
                 double* out, int64_t* evals, int brute);

/* Leave-one-out log likelihood for one fixed h, CPU branch of
 * kde_cuda_kdtr_tiled.cu:3300-3366:
 *   loo_j = sum_{i != j, d^2 < 9h^2} K_h(d) w_i e_i
 *   logL  = sum_j log(max(loo_j, EPSILONDENSITY))
 * ew == NULL means unit edge weights (edge correction off).  The caller
 * supplies e_i(h) (the reference recomputes them for every h). */
double orc_loo_loglik(int64_t n, const float* x, const float* y, const float* w,
                      const double* ew, float h, double* out_loo, int64_t* evals);

/* Full per-h evaluation as LogLikelihood() does it: edge weights at h
 * (when dist2 != NULL) then the LOO sum.  Returns logL; evals adds both
 * the edge-correction and the LOO pair counts. */
double orc_loglik_at(int64_t n, const float* x, const float* y, const float* w,
                     const double* dist2, const orc_grid* g, const float* mask,
                     float h, int64_t* evals);

/* Golden-section fixed-bandwidth search, kde_cuda_kdtr_tiled.cu:3044-3093
 * (bracket [h0/20, 2 h0], at most 30 iterations, returns the midpoint). */
float orc_mle_fixed_bandwidth(int64_t n, const float* x, const float* y, const float* w,
                              const double* dist2, const orc_grid* g, const float* mask,
                              float h0, int* iterations);

/* Density at the points themselves with per-source bandwidths:
 *   den_j = sum_{i, d_ij^2 < 9 h_i^2} K_{h_i}(d_ij) w_i e_i   (i = j included when self != 0)
 * hs == NULL -> fixed h.  ComputeFixedDensityAtPoints
 * (kde_cuda_kdtr_tiled.cu:3096-3133) with self, and the leave-one-out sums of
 * the adaptive LogLikelihood (CPU branch, :3604-3636) without. */
void orc_point_density(int64_t n, const float* x, const float* y, const float* w,
                       const double* ew, const float* hs, float h, int self,
                       double* out, int64_t* evals);

/* Adaptive bandwidths from a pilot density, kde_cuda_kdtr_tiled.cu:3581-3590:
 * gml = exp(mean log den0) (compGML, :3807-3814) and
 * hs_i = h (den0_i / gml)^alpha, stored as float. */
void orc_adaptive_bandwidths(int64_t n, const double* den0, float h, float alpha, float* hs);

/* Log likelihood of the adaptive bandwidths for (h, alpha), CPU branch of
 * LogLikelihood(h, alpha) (kde_cuda_kdtr_tiled.cu:3553-3650): edge weights at
 * the fixed h, pilot density with self, hs, edge weights at hs, and the
 * leave-one-out sum with per-source bandwidths.  dist2 == NULL: no edge
 * correction.  hs_out (optional) receives the bandwidths. */
double orc_loglik_adaptive(int64_t n, const float* x, const float* y, const float* w,
                           const double* dist2, const orc_grid* g, const float* mask,
                           float h, float alpha, float* hs_out);

/* Hooke-Jeeves search over (h, alpha), hooke_jeeves / hj_likelihood
 * (kde_cuda_kdtr_tiled.cu:3677-3785), with the reference's start
 * (alpha0 = -0.5, stepH = h0 / 10, stepA = 0.1, main :550-555), its float
 * step arithmetic and its bookkeeping of the five likelihoods, then the final
 * bandwidths of main (:566-572): pilot density at the optimum h with edge
 * weights at h, compGML, hs.  out: h_opt, alpha_opt, Lmax; hs (n floats). */
void orc_adaptive_search(int64_t n, const float* x, const float* y, const float* w,
                         const double* dist2, const orc_grid* g, const float* mask,
                         float h0, float* out3, float* hs, int* iterations);

/* Number of OpenMP threads the oracle uses (0 = library default). */
void orc_set_threads(int n);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
