/*
 * mgk.h — C ABI of the B200 (sm_100a) tiled fixed-bandwidth Gaussian KDE.
 *
 * The reference (mGPUKDE_tiled) has no plugin layer: its host driver launches
 * CUDA kernels that take POD structs by value holding raw device pointers
 * (SamplePoints, SamplePoints.h:9-17; AsciiRaster, AsciiRaster.h:9-33) and
 * calls host functions over them.  Each entry point below replaces one of
 * those launches or host functions; the citation says which.
 *
 * Conventions
 *  - Every function returns an int status: 0 (MGK_OK) or a negative MGK_ERR_*.
 *    Nothing calls exit(); mgk_ctx_last_error() gives the message.
 *  - Work is ordered on the context's CUDA stream (mgk_ctx_set_stream).
 *    Functions that return host-side results (counts, log likelihoods)
 *    synchronise that stream before returning.
 *  - Rasters are row-major with row 0 at the top, NoData passed through, as
 *    in the reference.  Cell centres: x = xll + (col + 0.5) cs,
 *    y = yll + (nrows - 0.5 - row) cs, computed in double and rounded to float
 *    (Utilities.h:13-14).
 *  - Device memory a context allocates counts against its HBM budget; a
 *    request beyond it fails with MGK_ERR_BUDGET and leaves the device usable.
 *  - One context per host thread.
 */
#ifndef MGK_H
#define MGK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGK_OK 0
#define MGK_ERR_INVALID (-1)   /* bad argument */
#define MGK_ERR_CUDA (-2)      /* CUDA runtime error */
#define MGK_ERR_BUDGET (-3)    /* HBM budget exceeded */
#define MGK_ERR_NO_DEVICE (-4) /* no CUDA device / wrong architecture */
#define MGK_ERR_TIMEOUT (-5)   /* a bounded device-side wait ran out */
#define MGK_ERR_IO (-6)        /* file read/write failure (host driver) */

/* Raster geometry: the fields of AsciiRaster (AsciiRaster.h:9-33) that the
 * path reads. */
typedef struct mgk_grid {
    int64_t ncols;
    int64_t nrows;
    float xll;
    float yll;
    float cs;
    float nodata;
} mgk_grid;

typedef struct mgk_ctx mgk_ctx;       /* device, stream, HBM budget, last error */
typedef struct mgk_points mgk_points; /* device-resident SamplePoints + per-point h, dist2, edge weights */
typedef struct mgk_raster mgk_raster; /* device-resident mask raster (AsciiRaster) */
typedef struct mgk_index mgk_index;   /* cell-binned point index (replaces KDtree/CUDA_KDTree) */

/* ---- context ---------------------------------------------------------- */

/* Replaces the device selection and per-GPU stream setup of main()
 * (kde_cuda_kdtr_tiled.cu:366-400).  hbm_budget_bytes = 0 means "free
 * memory at creation".  Fails with MGK_ERR_NO_DEVICE unless the device is
 * compute capability 10.x. */
int mgk_ctx_create(int device, uint64_t hbm_budget_bytes, mgk_ctx** out);
int mgk_ctx_destroy(mgk_ctx* ctx);
/* Use an external stream (cudaStream_t as void*); NULL = the context's own. */
int mgk_ctx_set_stream(mgk_ctx* ctx, void* cuda_stream);
int mgk_ctx_synchronize(mgk_ctx* ctx);
const char* mgk_ctx_last_error(const mgk_ctx* ctx);
uint64_t mgk_ctx_bytes_in_use(const mgk_ctx* ctx);
const char* mgk_status_string(int status);
/* Instrumentation (no reference counterpart; the reference prints wall-clock
 * phase timings, kde_cuda_kdtr_tiled.cu:994, 1521): number of kernels this
 * context has launched, and the device time in ms of the last density
 * kernel (CUDA events on the context stream around that one launch). */
uint64_t mgk_ctx_kernel_launches(const mgk_ctx* ctx);
float mgk_ctx_last_density_ms(const mgk_ctx* ctx);
/* Instrumentation of the last likelihood computation: an
 * mgk_loo_loglik_batch / golden-section step (the device time in ms of the
 * batch: CUDA events on the context stream around the edge weights, the
 * gather, the sums and the argmax), or a whole mgk_loglik_adaptive /
 * mgk_adaptive_bandwidths call (events around all of its work, host waits
 * included); and its algorithmic eval counts (edge-mask cells in the cutoff,
 * point pairs in the cutoff, summed over every likelihood evaluated).
 * No reference counterpart. */
float mgk_ctx_last_loo_ms(const mgk_ctx* ctx);
int mgk_ctx_last_loo_evals(const mgk_ctx* ctx, int64_t* edge_evals, int64_t* loo_evals);

/* ---- points (SamplePoints) --------------------------------------------- */

/* Host -> device copy of a point set; replaces AllocateDeviceSamplePoints +
 * CopyToDeviceSamplePoints (kde_cuda_kdtr_tiled.cu:1713-1805) and the
 * bandwidth upload (CopyToDeviceBandwidths).  w == NULL: unit weights.
 * h == NULL: a fixed bandwidth is given per call; else per-point h
 * (h_option -1, kde_cuda_kdtr_tiled.cu:413-421). */
int mgk_points_upload(mgk_ctx* ctx, int64_t n, const float* x, const float* y,
                      const float* w, const float* h, mgk_points** out);
/* Same over caller-owned device arrays (no copy; they must outlive the
 * handle).  dist2 / edge-weight storage is still allocated by the library. */
int mgk_points_wrap(mgk_ctx* ctx, int64_t n, const float* d_x, const float* d_y,
                    const float* d_w, const float* d_h, mgk_points** out);
int mgk_points_destroy(mgk_points* pts);
/* The points of src inside [xlo, xhi] x [ylo, yhi], in their input order, as
 * a new device point set (x, y and, when src has them, w and per-point h;
 * boundary distances and edge weights are computed afresh on it).  It is the
 * device form of the reference's halo filter ExtractSamplePointsCurTile
 * (kde_cuda_kdtr_tiled.cu:4672-4747): a rank of a multi-GPU study keeps the
 * points within 3h of its rows, whose densities need no others.  One read
 * back of the count synchronises the context stream. */
int mgk_points_select(mgk_ctx* ctx, const mgk_points* src, double xlo, double xhi, double ylo, double yhi,
                      mgk_points** out);
/* Number of points of a point set (NULL: 0).  No reference counterpart (the
 * reference reads SamplePoints.numberOfPoints). */
int64_t mgk_points_size(const mgk_points* pts);
/* Device pointers of a point set (any may be NULL on output when absent):
 * x, y, w, h (float), dist2 (double, squared distance to the boundary),
 * ew (float, edge-correction weight). */
int mgk_points_device_arrays(const mgk_points* pts, const float** x, const float** y,
                             const float** w, const float** h, const double** dist2,
                             const float** ew);
/* Device -> host copy of the per-point results (either may be NULL);
 * replaces ReformECWeights / CopyFromDevice* (kde_cuda_kdtr_tiled.cu:4589-4646). */
int mgk_points_download(mgk_points* pts, double* dist2, float* ew);

/* ---- rasters (AsciiRaster) -------------------------------------------- */

/* Host -> device mask raster; replaces AllocateDeviceAsciiRaster +
 * CopyToDeviceAsciiRaster (kde_cuda_kdtr_tiled.cu:2264-2373). */
int mgk_raster_upload(mgk_ctx* ctx, const mgk_grid* g, const float* mask, mgk_raster** out);
int mgk_raster_wrap(mgk_ctx* ctx, const mgk_grid* g, const float* d_mask, mgk_raster** out);
int mgk_raster_destroy(mgk_raster* r);

/* ---- boundary and distance --------------------------------------------- */

/* dMarkBoundary + MarkBoundary (kde_kernel_kdtr.cu:1209-1281,
 * kde_cuda_kdtr_tiled.cu:3956-3992): marks boundary cells of the mask and
 * keeps their centres with the raster.  n_boundary (optional, host) gets the
 * count. */
int mgk_mark_boundary(mgk_ctx* ctx, mgk_raster* mask, int64_t* n_boundary);
/* Optional copy of the boundary flags (uint8 per cell, row-major). */
int mgk_raster_boundary_download(mgk_raster* mask, uint8_t* out);
/* dCalcDist2Boundary + CalcDist2Boundary (kde_kernel_kdtr.cu:1285-1353,
 * kde_cuda_kdtr_tiled.cu:4072-4137): exact FP64 squared distance from every
 * point to the nearest boundary-cell centre (DBL_MAX when there is none).
 * Marks the boundary first if mgk_mark_boundary has not run. */
int mgk_boundary_dist(mgk_ctx* ctx, mgk_points* pts, mgk_raster* mask);
/* The same distances made exact only for points whose nearest boundary cell
 * lies within `reach` (coordinate units); the others get a value above
 * reach^2.  The distances matter only through the edge-weight short-circuit
 * (weight 1 when dist2 >= 9 h^2, kde_cuda_kdtr_tiled.cu:2704-2708), so a reach
 * of 3 h_max gives the same edge weights as mgk_boundary_dist at a fraction
 * of the search (points deep inside the study area skip it).  The calls that
 * read the distances (edge weights, likelihoods) check that the reach covers
 * 3h for every bandwidth they use and fail with MGK_ERR_INVALID otherwise;
 * the adaptive-bandwidth calls need mgk_boundary_dist.  No reference
 * counterpart (the reference computes every distance exactly, brute force). */
int mgk_boundary_dist_within(mgk_ctx* ctx, mgk_points* pts, mgk_raster* mask, double reach);

/* ---- edge correction --------------------------------------------------- */

/* CalcEdgeCorrectionWeights, both overloads (kde_kernel_kdtr.cu:117-265;
 * CPU twins kde_cuda_kdtr_tiled.cu:2694-2807): weight 1 when dist2 >= 9 h^2,
 * else 1 / sum over valid mask cells with d^2 < 9 h^2 of K_h(d) * cellArea.
 * h > 0: fixed bandwidth; h <= 0: the points' per-point h.  Requires
 * mgk_boundary_dist first (else MGK_ERR_INVALID).  evals (optional, host)
 * receives the number of in-cutoff (point, cell) pairs. */
int mgk_edge_weights(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask, float h,
                     int64_t* evals);
/* Sets every edge weight to 1 (edge correction off; InitdWeights,
 * kde_kernel_kdtr.cu:665-676). */
int mgk_edge_weights_unit(mgk_ctx* ctx, mgk_points* pts);

/* ---- cell-binned index -------------------------------------------------- */

/* Replaces BuildCPUKDtree + BuildGPUKDtree (kde_cuda_kdtr_tiled.cu:4241-4275,
 * CUDA_KDtree.cu:26-102) and the per-tile halo filter ExtractSamplePointsCurTile
 * (kde_cuda_kdtr_tiled.cu:4672-4747): points are counting-sorted (stable LSD
 * radix sort) into square bins of side bin_size (0 = chosen from h) and
 * stored bin-major with w * e folded in.  h > 0: fixed h; h <= 0: per-point h.
 * The index snapshots the points' current edge weights. */
int mgk_index_build(mgk_ctx* ctx, const mgk_points* pts, float h, float bin_size, mgk_index** out);
int mgk_index_destroy(mgk_index* idx);

/* ---- density ------------------------------------------------------------ */

/* KernelDesityEstimation_pPoints + InitCellDensities (kde_kernel_kdtr.cu:
 * 268-294, 461-574) for one tile: rows [row0, row0+nr) x cols [col0, col0+nc)
 * of the raster geometry g.  d_mask_tile: nr*nc floats, NoData cells are
 * passed through (NULL = every cell valid).  d_out: nr*nc floats, density of
 * valid cells (intensity, not probability).  evals (optional, host): number
 * of in-cutoff (point, cell) pairs (synchronises). */
int mgk_density_tile(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0,
                     int64_t col0, int64_t nr, int64_t nc, const float* d_mask_tile,
                     float* d_out, int64_t* evals);
/* Same with the plain FP64 form of the kernel (double throughout, no
 * compensation): the comparator the FP32-compensated kernel is measured
 * against. */
int mgk_density_tile_fp64(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0,
                          int64_t col0, int64_t nr, int64_t nc, const float* d_mask_tile,
                          float* d_out, int64_t* evals);

/* Same density as mgk_density_tile, for callers that cannot let the library
 * allocate device memory at call time (an application that reserves the GPU's
 * memory up front for its own allocator, or a running latency-critical loop
 * in which cudaMalloc/cudaFree, which may synchronise the device, are not
 * allowed).  It calls no cudaMalloc, cudaFree or other allocating routine:
 * its scratch (block counts, work items, FP64 partial sums of split blocks)
 * lives in one fixed file-scope device array of about 12.3 MiB that every GPU
 * loading the library holds until the process exits.  Limit: tiles of at most
 * 4096 x 4096 cells (MGK_ERR_INVALID beyond).  The first call on a device looks
 * up that array's device address (once per device).  Every call makes
 * ctx's device current for its duration (the caller's device is restored on
 * return) and waits on ctx's stream twice (the plan reads the block counts
 * back, and the call finishes before returning, because the next call reuses
 * the array), so it cannot be called while that stream is being captured.
 * All calls share the one array and keep the last call's contents: calls
 * that overlap on the GPU (other streams, other threads) race and must be
 * serialised by the caller.  No counterpart in the reference. */
int mgk_density_tile_noalloc(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0,
                             int64_t col0, int64_t nr, int64_t nc, const float* d_mask_tile,
                             float* d_out);

/* Several density tiles in one launch (continuous batching of small jobs):
 * each job is one tile of one index over its own raster, as for
 * mgk_density_tile.  The tiles are planned independently, so each result is
 * bitwise the result of mgk_density_tile on that tile alone.  evals
 * (optional, host, njobs entries): algorithmic pair counts per job (the
 * counting kernel variant runs when given).  No reference counterpart (the
 * reference runs one tile at a time, kde_cuda_kdtr_tiled.cu:1233-1517). */
typedef struct mgk_tile_job {
    const mgk_index* index;
    mgk_grid grid;                 /* the raster the tile belongs to */
    int64_t row0, col0, nrows, ncols;
    const float* d_mask;           /* device, nrows x ncols row-major, or NULL */
    float* d_out;                  /* device, nrows x ncols row-major */
} mgk_tile_job;
int mgk_density_tiles(mgk_ctx* ctx, int njobs, const mgk_tile_job* jobs, int64_t* evals);

/* Out-of-core density: the raster in row-major tiles of tile_side^2 cells,
 * each handed to `sink` (on a library thread, in tile order, after its data
 * is final) while the GPU computes the next ones; mask tiles (optional) come
 * from `mask_src` (on the calling thread) into an nrows x ncols buffer.
 * done (optional, one byte per tile, row-major tile order): tiles to skip,
 * for resuming an interrupted run.  A nonzero return from a callback stops
 * the run with MGK_ERR_IO; tiles already given to the sink stay valid.
 * evals (optional): algorithmic pair count of the tiles computed.  The
 * reference's tile loop is kde_cuda_kdtr_tiled.cu:1233-1517 (GeoTIFF reads
 * and writes per tile, GeoTIFF.cpp:494-575). */
typedef int (*mgk_tile_source)(void* user, int64_t tile, int64_t row0, int64_t col0, int64_t nrows,
                               int64_t ncols, float* mask_out);
typedef int (*mgk_tile_sink)(void* user, int64_t tile, int64_t row0, int64_t col0, int64_t nrows,
                             int64_t ncols, const float* density);
int mgk_density_stream(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t tile_side,
                       mgk_tile_source mask_src, void* src_user, mgk_tile_sink sink, void* sink_user,
                       const uint8_t* done, int64_t* evals);
/* A ready-made sink: copies each tile into a whole host raster;
 * sink_user points to an mgk_copy_target. */
typedef struct mgk_copy_target {
    float* base;                   /* host, nrows x ncols row-major */
    int64_t ncols;
} mgk_copy_target;
int mgk_copy_sink(void* target, int64_t tile, int64_t row0, int64_t col0, int64_t nrows, int64_t ncols,
                  const float* density);

/* ---- bandwidth selection ---------------------------------------------- */

/* Batched LogLikelihood (kde_cuda_kdtr_tiled.cu:3214-3299) over nh fixed
 * bandwidths in one pass: for each h, edge weights at h (when mask != NULL;
 * needs mgk_boundary_dist), then
 *   logL(h) = sum_j log(max(sum_{i != j, d^2 < 9h^2} K_h(d) w_i e_i(h), 1e-14f))
 * reduced in FP64.  logL: nh doubles (host).  argmax (optional, host): index
 * of the largest logL. */
int mgk_loo_loglik_batch(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask,
                         const float* h_grid, int nh, double* logL, int* argmax);
/* Multi-GPU form of mgk_loo_loglik_batch, one process per GPU.  The
 * reference's LogLikelihood splits the points over its GPUs (each GPU
 * computes the edge weights of Points[i].start..end and the densities they
 * scatter) and merges through host memory (ReformECWeights,
 * ReformGPUDensities, ReductionSumGPU; kde_cuda_kdtr_tiled.cu:3223-3297).
 * Here rank `part` of `nparts` (c = ceil(n / nparts)):
 *  1. mgk_loo_share_edge_weights: e_i(h_k) of its points
 *     [part c, min(n, (part + 1) c)) for every h of h_grid, into its chunk of
 *     d_ew_all (device, nparts * nh * c floats; chunk `part` holds nh rows of
 *     c floats: e of point part c + j at h_k is d_ew_all[part nh c + k c + j]).
 *     Needs mgk_boundary_dist.  The caller then all-gathers the chunks (one
 *     ncclAllGather of nh c floats per rank, in place).
 *  2. mgk_loo_share_loglik: for every h_k, the FP64 sum of
 *     log(max(loo_j(h_k), 1e-14f)) over this rank's share of the queries
 *     (every point is a source): the query groups
 *     [part G / nparts, (part + 1) G / nparts) of h_k's index, G = ceil(n / 128)
 *     groups of 128 points in Z-order of the index bins.  d_ew_all: the
 *     gathered edge weights, or NULL without edge correction.  The shares of
 *     parts 0 .. nparts-1 cover every query exactly once per h, so the sum of
 *     partial_logL over ranks (one all-reduce of nh doubles) is logL(h); its
 *     argmax is the bandwidth.  evals (optional): this share's pair count. */
int mgk_loo_share_edge_weights(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask, const float* h_grid,
                               int nh, int part, int nparts, float* d_ew_all, int64_t* evals);
int mgk_loo_share_loglik(mgk_ctx* ctx, mgk_points* pts, const float* h_grid, int nh, int part, int nparts,
                         const float* d_ew_all, double* partial_logL, int64_t* evals);
/* MLE_FixedBandWidth (kde_cuda_kdtr_tiled.cu:3044-3093): golden-section
 * search on [h0/20, 2 h0], at most 30 iterations, two logL evaluations per
 * iteration (each one batched launch of nh=2); returns the bracket midpoint. */
int mgk_mle_fixed_bandwidth(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask, float h0,
                            float* h_opt, int* iterations);
/* LogLikelihood with adaptive bandwidths (kde_cuda_kdtr_tiled.cu:3553-3650,
 * the CPU branch of the h_option 2 likelihood): edge weights at h, pilot
 * density at every point (itself included), hs_i = h (den_i / gml)^alpha with
 * gml the geometric mean of the pilot densities (compGML, :3655-3672), edge
 * weights at hs, then
 *   logL = sum_j log(max(sum_{i != j, d^2 < 9 hs_i^2} K_{hs_i}(d) w_i e_i(hs), 1e-14f)).
 * mask NULL: no edge correction (mask != NULL needs mgk_boundary_dist).
 * Leaves hs in the points' per-point bandwidths (points that wrap caller
 * memory get a buffer of their own; the caller's h array is not written). */
int mgk_loglik_adaptive(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask, float h, float alpha,
                        double* logL);
/* h_option 2 (main, kde_cuda_kdtr_tiled.cu:548-573): Hooke-Jeeves search
 * (hooke_jeeves / hj_likelihood, :3677-3785) of (h, alpha) from (h0, -0.5)
 * with steps h0/10 and 0.1, at most 30 iterations, maximising
 * mgk_loglik_adaptive; then the bandwidths of the optimum, hs_i = h (den_i /
 * gml)^alpha, from the pilot density at the fixed h.  hs are left in the
 * points' per-point bandwidths and copied to hs_out (host, n floats; may be
 * NULL).  The points' edge weights are invalidated: compute them at hs
 * (mgk_edge_weights with h = 0) before the density.  h_opt, alpha_opt, lmax
 * (the largest logL seen, held as a float like the reference's), iterations:
 * host, each may be NULL. */
int mgk_adaptive_bandwidths(mgk_ctx* ctx, mgk_points* pts, const mgk_raster* mask, float h0, float* h_opt,
                            float* alpha_opt, double* lmax, int* iterations, float* hs_out);
/* Rule-of-thumb bandwidth (kde_cuda_kdtr_tiled.cu:64-68, 1563-1595), host
 * arithmetic identical to the reference's. */
float mgk_rule_of_thumb(int64_t n, const float* x, const float* y, const float* w);

/* ---- tuning ------------------------------------------------------------ */
/* Launch-shape settings of a context.  bin_factor: index bin side / h when
 * mgk_index_build gets bin_size 0 (default 0.5); split_waves: the density
 * plan splits blocks into work items of at most total / (resident CTAs x
 * split_waves) candidates (default 4); tile_side: density tile side used by
 * mgk_kde_raster when its tile argument is 0 (0: the whole raster). */
typedef struct mgk_tuning {
    float bin_factor;
    int32_t split_waves;
    int64_t tile_side;
    float density_ms;              /* autotune: time of the chosen bin side on its sample windows */
    int32_t from_cache;            /* autotune: 1 when read from the cache file */
} mgk_tuning;
int mgk_ctx_get_tuning(const mgk_ctx* ctx, mgk_tuning* out);
int mgk_ctx_set_tuning(mgk_ctx* ctx, const mgk_tuning* t);
/* Measures the bin factor (0.5, 0.75, 1, 1.25 x h, on four 1024^2 sample
 * windows of g) and, for rasters above 4096 cells a side, the streamed tile
 * side (2048, 4096, 8192 over the same central area) for these points and h,
 * applies them to ctx and appends them to cache_file (optional) under a key
 * of GPU, point count, h in cells and point density; a later call with a
 * matching key reads the file instead of measuring.  No reference
 * counterpart (the reference's launch shapes are compile-time constants). */
int mgk_autotune(mgk_ctx* ctx, const mgk_points* pts, float h, const mgk_grid* g, const char* cache_file,
                 mgk_tuning* out);

/* ---- serving loop ------------------------------------------------------ */
/* Two threads, each with its own context on `device` (HBM budget as for
 * mgk_ctx_create), serve whole fixed-h KDE requests.  The preparation thread
 * admits requests by free slots (max_active) and their estimated device
 * footprint within the budget, uploads and indexes them (their points,
 * index and tiles are its context's memory, resident while a request is
 * active) and frees them when they finish.  The worker thread runs each
 * tick as one density launch over the next tile (tile_side^2 cells) of
 * every active request, so requests that arrive while others run join the
 * next tick (continuous batching); its context holds only per-tick plan
 * scratch.  A request's raster is bitwise the same alone or in a mix.  No
 * reference counterpart (the reference runs one study per process). */
typedef struct mgk_server mgk_server;
typedef struct mgk_request {
    int64_t n;
    const float *x, *y, *w;      /* host, n each; w may be NULL */
    float h;                     /* fixed bandwidth */
    mgk_grid grid;               /* density raster */
    const float* mask;           /* host density mask (NoData passthrough) or NULL */
    int edge;                    /* edge correction on the edge mask below */
    mgk_grid edge_grid;
    const float* edge_mask;      /* host */
    float* out;                  /* host, grid.nrows x grid.ncols */
} mgk_request;
typedef struct mgk_result {
    int status;                  /* MGK_OK or the failing call's status */
    int64_t evals;               /* density + edge-correction pairs in the cutoff */
    double queue_ms, run_ms, total_ms;
} mgk_result;
typedef struct mgk_serve_info {
    uint64_t ticks, tiles, max_batch, completed, queued, active, reserved_bytes, device_bytes;
} mgk_serve_info;
int mgk_serve_create(int device, uint64_t hbm_budget_bytes, int64_t tile_side, int max_active,
                     mgk_server** out);
/* Queues a request (its host buffers must stay valid until it completes). */
int mgk_serve_submit(mgk_server* srv, const mgk_request* req, uint64_t* ticket);
/* done = 1 and the result once finished (the ticket is then released). */
int mgk_serve_poll(mgk_server* srv, uint64_t ticket, int* done, mgk_result* res);
/* Blocks until the request finishes (its status is returned) or timeout_s
 * passes (MGK_ERR_TIMEOUT, the ticket stays valid). */
int mgk_serve_wait(mgk_server* srv, uint64_t ticket, double timeout_s, mgk_result* res);
int mgk_serve_stats(mgk_server* srv, mgk_serve_info* out);
/* Finishes the queued and active requests, then stops both threads. */
int mgk_serve_destroy(mgk_server* srv);

/* ---- whole path from host buffers ------------------------------------- */

/* The GPU section of main() (kde_cuda_kdtr_tiled.cu:877-1521) for one raster
 * held in host memory: upload, boundary + distance + edge weights (when
 * edge_correction), index, tiled density, download.  h_pp == NULL: fixed h.
 * dens_mask == NULL: every density cell valid.  out_density: host,
 * nrows*ncols of dens_g.  out_ew (optional): per-point edge weights.
 * evals (optional): density + edge-correction in-cutoff pairs. */
int mgk_kde_raster(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* w,
                   const float* h_pp, float h, int edge_correction, const mgk_grid* edge_g,
                   const float* edge_mask, const mgk_grid* dens_g, const float* dens_mask,
                   int64_t tile_side, float* out_density, float* out_ew, int64_t* evals);
/* The same path for rows [row0, row0 + nrows) of dens_g only: one rank's
 * share of a study split over GPUs by rows, with no exchange between ranks
 * (the densities of these rows need only the points within 3h of them).
 * The reference splits the points instead and sums whole tiles from every GPU
 * through host memory (kde_cuda_kdtr_tiled.cu:1320-1351, ReformGPUAsciiRaster
 * :2468-2567).  All n points are passed; after the upload only those within
 * 3 h_max of the rows are kept (mgk_points_select), so the boundary
 * distances, edge weights and index cover only them.  dens_mask_rows and
 * out_rows: host, nrows x ncols, the rows' part of the raster.  evals
 * (optional): the rows' density pairs plus the edge-correction pairs of the
 * kept points. */
int mgk_kde_raster_rows(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* w,
                        const float* h_pp, float h, int edge_correction, const mgk_grid* edge_g,
                        const float* edge_mask, const mgk_grid* dens_g, int64_t row0, int64_t nrows,
                        const float* dens_mask_rows, int64_t tile_side, float* out_rows, int64_t* evals);

#ifdef __cplusplus
}
#endif
#endif /* MGK_H */
