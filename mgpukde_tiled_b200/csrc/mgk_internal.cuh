// Internal declarations shared by the CUDA translation units of libmgk.
#pragma once
#include <cstring>

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <string>

#include "../../include/mgk.h"

// ---- constants of the reference (Utilities.h) -----------------------------
// TWO_PI is a float constant in the reference (Utilities.h:8).
#define MGK_TWO_PI_F 6.2831853071795862f
// EPSILONDENSITY (Utilities.h:20), a float constant.
#define MGK_EPS_DENSITY_F 0.00000000000001f
// CUT_OFF_FACTOR (Utilities.h:27): the kernel is zero for d^2 >= 9 h^2.
#define MGK_CUT 9.0
#define MGK_LOG2E 1.4426950408889634
#define MGK_LN2F 0.69314718055994531f

// ---- host-side objects -----------------------------------------------------
struct mgk_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    std::atomic<uint64_t> in_use{0};  // read by other threads (serving statistics)
    std::string last_error;
    // small pinned/device scratch for scalar results
    unsigned long long* d_counter = nullptr;  // 8 counters
    unsigned long long* h_counter = nullptr;  // pinned mirror
    double* d_sum = nullptr;                  // 256 doubles
    double* h_sum = nullptr;                  // pinned mirror
    // mapped page-locked staging of plans and counts (mgk_host_stage), in
    // kStageSlots independent slots; h_stage[i] and d_stage[i] address the same
    // bytes.  Slot 3 holds the bit-packed density mask of mgk_kde_raster.
    static constexpr int kStageSlots = 4;
    void* h_stage[kStageSlots] = {};
    void* d_stage[kStageSlots] = {};
    size_t h_stage_bytes[kStageSlots] = {};
    std::multimap<size_t, void*> pool;        // cached device blocks by size class
    uint64_t launches = 0;                    // kernels launched by this context
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    float last_density_ms = 0.0f;
    int64_t last_loo_evals[2] = {0, 0};  // edge and LOO evals of the last LOO batch run
    float last_loo_ms = 0.0f;
    // tuning (mgk_autotune / mgk_ctx_set_tuning)
    float bin_factor = 0.5f;   // default index bin side / h (fastest of 0.5-1.25 on the 1e6-point raster)
    int split_waves = 4;       // density work items per resident CTA slot (4 of 2-32 fastest on the C1 raster)
    int64_t tile_side = 0;     // streamed tile side (0: whole raster when it fits)
};

#define MGK_COUNT_LAUNCH(ctx, k) ((ctx)->launches += (k))

struct mgk_points {
    mgk_ctx* ctx = nullptr;
    int64_t n = 0;
    float *x = nullptr, *y = nullptr, *w = nullptr, *h = nullptr;
    bool owns_xywh = false;
    bool owns_h = false;  // h allocated by the adaptive search on points that do not own x/y/w/h
    double* dist2 = nullptr;
    bool has_dist2 = false;
    // dist2 is exact for the points whose nearest boundary cell lies within
    // dist2_cap (coordinate units); the others hold a value above dist2_cap^2
    double dist2_cap = 0.0;
    float* ew = nullptr;
    bool has_ew = false;
};

struct mgk_raster {
    mgk_ctx* ctx = nullptr;
    mgk_grid g{};
    float* mask = nullptr;
    bool owns = false;
    uint8_t* boundary = nullptr;  // per cell
    float2* bcells = nullptr;     // boundary-cell centres, binned
    int* bstart = nullptr;        // bin offsets into bcells (nbins + 1)
    int* bnear = nullptr;         // per bin: first ring index holding a non-empty bin
    double* bub = nullptr;        // per bin: upper bound of the nearest-cell d^2 of its points
    int* cstart = nullptr;        // per bin: offsets of its candidate list in cand (nbins + 1)
    float2* cand = nullptr;       // candidate boundary-cell centres, bin by bin
    int64_t ncand = 0;
    double cand_cap = -1.0;       // the lists hold the cells within this reach of each bin (< 0: no lists)
    int bnx = 0, bny = 0;         // boundary bins per row / column
    int64_t nbins = 0;
    int64_t nb = 0;
    bool marked = false;
    // valid-cell runs per row: runs[run_start[r] .. run_start[r+1]) = [a, b)
    int64_t* run_start = nullptr;  // nrows + 1
    int2* runs = nullptr;
    int64_t nruns = 0;
    bool has_runs = false;
};

// One point of the bin-major index (32 B, one bulk copy moves whole records).
// Coordinates are split on a global quantum q = 2^-qexp: x = xh + xl exactly,
// xh a multiple of q, |xl| <= q/2.  Cell centres are split on the same
// quantum, so xh - cxh is exact in FP32 and the distance is recovered
// exactly as a float pair.  wk = w * e (fixed h) or w * e / (h^2 TWO_PI)
// (per-point h); k2h + k2l = log2(e) / (2 h^2) and hh = h*h (float product)
// for per-point h, zero otherwise.
struct __align__(16) MgkPt {
    float xh, yh, xl, yl;
    float wk, k2h, k2l, hh;
};

struct mgk_index {
    mgk_ctx* ctx = nullptr;
    int64_t n = 0;
    bool varh = false;
    int qexp = 0;  // coordinate quantum 2^-qexp
    // fixed-h constants (double): h^2 as the reference forms it, 9 h^2,
    // log2(e)/(2 h^2), 1/(h^2 TWO_PI), 3 h
    float h = 0.0f;
    double h2 = 0, cut_d2 = 0, k2 = 0, k0 = 0, reach = 0;
    // bin grid
    double ox = 0, oy = 0, side = 1;
    int64_t nbx = 1, nby = 1;
    int32_t* bin_start = nullptr;  // nbx*nby + 1
    // bin-major point data
    MgkPt* pts = nullptr;
    int32_t* perm = nullptr; // sorted position -> input index
    uint64_t bytes = 0;
};

// ---- helpers ---------------------------------------------------------------
int mgk_fail(mgk_ctx* ctx, int status, const std::string& msg);
int mgk_cuda_fail(mgk_ctx* ctx, cudaError_t e, const char* what);
int mgk_alloc(mgk_ctx* ctx, void** p, size_t bytes);
// Mapped page-locked host memory of at least `bytes` owned by the context
// (grown on demand, previous contents not kept): *host and *dev address the
// same bytes.  Kernels read and write it directly over the bus, so small
// per-launch tables and flags need no copy-engine transfer and never queue
// behind large copies that other streams have in flight.  One user at a time:
// kernels using it must have finished before the next call.
int mgk_host_stage(mgk_ctx* ctx, size_t bytes, void** host, void** dev);
// The same for staging slot `slot` (0 is the one mgk_host_stage uses); plans
// that are alive at the same time use different slots.
int mgk_host_stage_slot(mgk_ctx* ctx, int slot, size_t bytes, void** host, void** dev);
void mgk_free(mgk_ctx* ctx, void* p, size_t bytes);

#define MGK_CHECK_CUDA(ctx, expr)                                   \
    do {                                                            \
        cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return mgk_cuda_fail(ctx, e_, #expr); \
    } while (0)

#define MGK_CHECK_LAUNCH(ctx, name)                                   \
    do {                                                              \
        cudaError_t e_ = cudaGetLastError();                          \
        if (e_ != cudaSuccess) return mgk_cuda_fail(ctx, e_, name);   \
    } while (0)

// ---- device helpers --------------------------------------------------------
__device__ __host__ __forceinline__ int64_t mgk_min64(int64_t a, int64_t b) { return a < b ? a : b; }
__device__ __host__ __forceinline__ int64_t mgk_max64(int64_t a, int64_t b) { return a > b ? a : b; }

__device__ __forceinline__ float mgk_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 2^-a for a double exponent a >= 0, to about the accuracy of ex2.approx:
// the exponent is split into float hi + lo and the lo part applied to first
// order (2^-(hi+lo) = 2^-hi (1 - lo ln2 + ...), |lo| <= 2^-24 hi).
__device__ __forceinline__ float mgk_exp2_neg(double a) {
    const float ah = __double2float_rn(a);
    const float al = __double2float_rn(a - (double)ah);
    const float e = mgk_ex2(-ah);
    return fmaf(-al * MGK_LN2F, e, e);
}

// 2^-a for 0 <= a < 120, without the special-function unit: a = n + f with
// n = rint(a), |f| <= 1/2 (Cody-Waite reduction), e^t for t = -f ln 2 from its
// Taylor series to degree 8 (truncation below 2.1e-10 relative for
// |t| <= ln2/2), Horner in FMA, then scaled by 2^-n through the exponent
// bits.  Its rounding errors have no common sign across inputs, so sums of
// many terms carry no systematic bias (used where millions of terms feed one
// logarithm sum).
__device__ __forceinline__ float mgk_exp2_neg_poly(float a) {
    const float n = rintf(a);
    const float t = __fmul_rn(__fsub_rn(n, a), MGK_LN2F);
    float p = 2.4801587301587302e-05f;  // 1/8!
    p = __fmaf_rn(p, t, 1.9841269841269841e-04f);  // 1/7!
    p = __fmaf_rn(p, t, 1.3888888888888889e-03f);  // 1/6!
    p = __fmaf_rn(p, t, 8.3333333333333333e-03f);  // 1/5!
    p = __fmaf_rn(p, t, 4.1666666666666667e-02f);  // 1/4!
    p = __fmaf_rn(p, t, 1.6666666666666667e-01f);  // 1/3!
    p = __fmaf_rn(p, t, 0.5f);
    p = __fmaf_rn(p, t, 1.0f);
    p = __fmaf_rn(p, t, 1.0f);
    return __fmul_rn(p, __int_as_float((127 - (int)n) << 23));
}

// Cell centres as the reference computes them (Utilities.h:13-14): double
// arithmetic, stored to float.
__device__ __host__ __forceinline__ float mgk_cell_x(double xll, double cs, int64_t col) {
    return (float)(xll + ((double)col + 0.5) * cs);
}
__device__ __host__ __forceinline__ float mgk_cell_y(double yll, double cs, int64_t nrows, int64_t row) {
    return (float)(yll + ((double)nrows - 0.5 - (double)row) * cs);
}

// Exact squared distance of two float positions with the rounding of the
// FP64 oracle (products and sum each rounded once, never fused).
__device__ __forceinline__ double mgk_d2_exact(float x0, float y0, float x1, float y1) {
    const double dx = __dsub_rn((double)x1, (double)x0);
    const double dy = __dsub_rn((double)y1, (double)y0);
    return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
}

// Splits a float coordinate on the quantum 2^-qexp: hi = nearest multiple,
// lo = remainder, both exact floats (|v| < 2^(22 - qexp) assumed).
// 2^k for a double exponent in the normal range (|k| < 1000), from its bits.
__device__ __host__ __forceinline__ double mgk_pow2(int k) {
    const unsigned long long b = (unsigned long long)(1023 + k) << 52;
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}
__device__ __host__ __forceinline__ void mgk_qsplit(float v, int qexp, float& hi, float& lo) {
    // scaling by powers of two is exact, so multiplying by 2^-qexp is the
    // division by 2^qexp
    hi = (float)(rint((double)v * mgk_pow2(qexp)) * mgk_pow2(-qexp));
    lo = (float)((double)v - (double)hi);
}

// h^2 exactly as the reference's CPU path forms it: float product widened.
__device__ __host__ __forceinline__ double mgk_h2(float h) {
    const float hh = h * h;
    return (double)hh;
}

// ---- kernels launched across translation units ------------------------------
int mgk_launch_index_build(mgk_ctx* ctx, const mgk_points* pts, float h, float bin_size, mgk_index* idx);
// The index records' weights from the points' current edge weights (an index
// built before the edge weights were known), stream-ordered on ctx->stream.
int mgk_index_refresh_weights(mgk_ctx* ctx, mgk_index* idx, const mgk_points* pts);
// d_order[k] = position of the k-th record of idx in Z-order of the bins (n entries, device).
int mgk_index_zorder(mgk_ctx* ctx, const mgk_index* idx, int32_t* d_order);
int mgk_launch_density(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0,
                       int64_t col0, int64_t nr, int64_t nc, const float* d_mask, float* d_out,
                       unsigned long long* d_evals, bool fp64);
int mgk_launch_density_jobs(mgk_ctx* ctx, int njobs, const mgk_tile_job* jobs, unsigned long long* d_evals);
// mgk_launch_density in two halves, so a caller can put its own copies
// between the plan (which synchronises the context stream and uploads the
// work list) and the kernels: prepare plans and uploads; execute launches,
// waits and releases the plan (also on failure); discard releases an unrun
// plan.  One plan at a time per context (the work list shares the context's
// page-locked staging).  A tile with no cells gives a null plan, which
// execute accepts.
struct mgk_dplan;
int mgk_density_prepare(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                        int64_t nr, int64_t nc, const float* d_mask, float* d_out, unsigned long long* d_evals,
                        bool fp64, mgk_dplan** out);
int mgk_density_execute(mgk_ctx* ctx, mgk_dplan* plan);
void mgk_density_discard(mgk_ctx* ctx, mgk_dplan* plan);
// A tile pipeline that plans tile k + 1 while tile k computes, all on one
// stream: counts_launch queues the counting kernel of a tile into staging
// slot `slot` (it leaves the shared staging-wait flag alone: the caller
// zeroes it once and reads it at the end); once that kernel has finished,
// plan_counted builds the plan from the counts into the same slot; launch
// queues the plan's kernels on stream s without waiting; discard releases the
// plan after its kernels have finished.
int mgk_density_counts_launch(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                              int64_t nr, int64_t nc, int slot, cudaStream_t s);
int mgk_density_plan_counted(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                             int64_t nr, int64_t nc, const float* d_mask, float* d_out, unsigned long long* d_evals,
                             int slot, mgk_dplan** out);
int mgk_density_launch_plan(mgk_ctx* ctx, mgk_dplan* plan, cudaStream_t s);
// The plan of rows/columns of a tile from per-block candidate counts in host
// memory (block-row major, ceil(nc / 128) per block row; e.g. a slice of one
// count of a larger tile whose block rows it shares); tables into `slot`.
int mgk_density_plan_from_counts(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                                 int64_t nr, int64_t nc, const int64_t* counts, const float* d_mask, float* d_out,
                                 unsigned long long* d_evals, int slot, mgk_dplan** out);
// Host view of the counts mgk_density_counts_launch wrote into `slot`.
const int64_t* mgk_density_counts_host(mgk_ctx* ctx, int slot);
// Copies a plan's work list from its staging slot to device memory on `s`
// now (mgk_density_launch_plan then skips that copy); the slot may be
// rewritten once this copy has run.
int mgk_density_stage(mgk_ctx* ctx, mgk_dplan* plan, cudaStream_t s);
// mgk_density_launch_plan with the merge of split blocks (if any) on
// s_merge, after the density on s (event ev); *merged_on_s_merge tells where
// the plan's last kernel went.
int mgk_density_launch_split(mgk_ctx* ctx, mgk_dplan* plan, cudaStream_t s, cudaStream_t s_merge, cudaEvent_t ev,
                             bool* merged_on_s_merge);
// The plan's density kernel sets *flag = 1 when its last CTA starts.
void mgk_density_set_tail_flag(mgk_dplan* plan, unsigned* flag);
// The plan's kernels read the tile's NoData mask as bits (device, 1 = valid,
// row r at byte r * stride, column c at bit c % 8 of byte c / 8) instead of floats.
void mgk_density_set_mask_bits(mgk_dplan* plan, const unsigned char* bits, int64_t stride);
int mgk_launch_mark_boundary(mgk_ctx* ctx, mgk_raster* r);
int mgk_raster_runs(mgk_ctx* ctx, mgk_raster* r);
int mgk_launch_dist2(mgk_ctx* ctx, mgk_points* p, mgk_raster* r, double cap);
int mgk_launch_edge_weights(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* hpp,
                            float h, const double* dist2, const mgk_raster* r, float* ew_out,
                            unsigned long long* d_evals);
int mgk_launch_edge_weights_multi(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* hpp,
                                  float hfix, const float* d_hgrid, int nh, const double* dist2,
                                  const mgk_raster* r, float* ew_out, int64_t ew_stride,
                                  unsigned long long* d_evals);

// Halo selection (index.cu): points of src inside a rectangle, input order.
// With dst == NULL: counts them into *count (d_scratch holds the per-tile
// offsets for the second call, mgk_points_select_scratch(n) unsigned).
int mgk_launch_points_select(mgk_ctx* ctx, const mgk_points* src, double xlo, double xhi, double ylo, double yhi,
                             unsigned* d_scratch, int64_t* count, mgk_points* dst);
int64_t mgk_points_select_scratch(int64_t n);

// Batched leave-one-out likelihood (loo.cu).
struct mgk_loo_batch;
int mgk_loo_batch_create(mgk_ctx* c, const mgk_points* p, const mgk_raster* r, float h_lo, float h_hi, int nh,
                         mgk_loo_batch** out);
int mgk_loo_batch_create_share(mgk_ctx* c, const mgk_points* p, const mgk_raster* r, float h_lo, float h_hi,
                               int nh, int part, int nparts, const float* ew_ext, int64_t ew_chunk,
                               mgk_loo_batch** out, bool replay = true);
int mgk_loo_batch_run(mgk_loo_batch* B, const float* hs, double* logl, int* best, int64_t* edge_evals,
                      int64_t* loo_evals);
void mgk_loo_batch_destroy(mgk_loo_batch* B);
