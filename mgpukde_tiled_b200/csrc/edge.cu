// Exact edge-correction weights (Diggle 1985).
//
// CalcEdgeCorrectionWeights (kde_kernel_kdtr.cu:117-189 fixed h, :192-265
// per-point h) and EdgeCorrectionWeightsExact (kde_cuda_kdtr_tiled.cu:2694-2807):
//   e_p = 1                                  if dist2_p >= 9 h^2
//   e_p = 1 / sum_{valid c, d^2 < 9h^2} K_h(d) cellArea   otherwise
// over the reference's NARROW row/column window (a superset of the 3h disc).
//
// The Gaussian factorises over the raster, K ~ exp(-dx^2/2h^2) exp(-dy^2/2h^2),
// and for one row the in-cutoff cells are one contiguous column interval:
// the FP64 test fl(fl(dx^2) + dy^2) < 9h^2 is monotone in |dx| and the cell
// centres are monotone in the column.  So per (point, h), with the column
// factors' prefix sums Q over the window,
//   sum = sum_rows exp(-dy^2/2h^2) * sum_{valid runs of the row} (Q[b] - Q[a])
// where [a, b) is a run of valid cells clipped to the row's in-cutoff
// interval.  The interval ends are found with the oracle's exact FP64 test
// (an estimate from sqrt(9h^2 - dy^2), verified, with a binary search when the
// estimate misses), so the summed cell set and the eval count are exactly the
// reference's.  Work per (point, h) is O(window width + window height) rather
// than O(width x height); the sums are FP64, the factors FP64 (per-point h)
// or FP32 to about 1e-7 (fixed h, edge_factor).
//
// One warp per point: the lanes build the prefix table of a chunk of up to
// 1024 window columns in shared memory (a contiguous segment per lane and a
// warp scan of the segment totals), then take the window rows in turn.  A
// list of bandwidths is handled in one launch (the LOO bandwidth search needs
// e_p(h) for every candidate h); the weights for h_k go to row k of the
// output.
#include <algorithm>

#include "mgk_internal.cuh"

namespace {

constexpr int kEdgeWarps = 4;     // warps per CTA
constexpr int kEdgeChunk = 1024;  // window columns per prefix table

struct EdgeParams {
    int64_t n;
    const float* x;
    const float* y;
    const float* hpp;    // per-point bandwidths (nh = 1) or null
    const float* hgrid;  // device bandwidth list (nh entries) or null: use hfix
    float hfix;
    int nh;
    const double* dist2;  // may be null: no short-circuit
    mgk_grid g;
    const int64_t* run_start;
    const int2* runs;
    float* ew;  // [nh][ew_stride]
    int64_t ew_stride;
    unsigned long long* evals;
    const int* list;        // with nh = 1: the points within 3h of the boundary, else null (all points)
    const int* list_count;  // its length (device)
};

// One bandwidth with boundary distances: the weight of a point 3h or more
// from the boundary is 1 (a coalesced pass); the others are listed (warp-
// aggregated appends, in no fixed order: each weight depends on its point
// alone) for the integral kernel.
template <bool VARH>
__global__ void k_edge_near(EdgeParams E, int* __restrict__ list, int* __restrict__ count) {
    const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    bool near = false;
    if (p < E.n) {
        const float hp = VARH ? E.hpp[p] : (E.hgrid ? E.hgrid[0] : E.hfix);
        if (E.dist2[p] >= MGK_CUT * mgk_h2(hp)) E.ew[p] = 1.0f;
        else near = true;
    }
    const unsigned b = __ballot_sync(0xffffffffu, near);
    if (!b) return;  // warp-uniform
    int base = 0;
    if (lane == 0) base = atomicAdd(count, __popc(b));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (near) list[base + __popc(b & ((1u << lane) - 1u))] = (int)p;
}

__device__ __forceinline__ int64_t trunc_index(double v) {
    v = fmin(fmax(v, -1.0e15), 1.0e15);
    return (int64_t)trunc(v);
}

__device__ __forceinline__ int64_t clamp_index(double v, int64_t lo, int64_t hi) {
    v = fmin(fmax(v, (double)lo), (double)hi);
    return (int64_t)v;
}

__device__ __forceinline__ double cell_xd(const mgk_grid& g, int64_t c) { return (double)mgk_cell_x(g.xll, g.cs, c); }

// exp(-d2 / 2h^2) for d2 within the cutoff (exponent <= 4.5).  Fixed h:
// 2^-(d2 k2) with the exponent in FP64, split into a float pair, 2^-hi by
// the unbiased FP32 polynomial and a first-order correction for the low part
// (relative error about 1e-7; the weights then meet the 1e-6 density and
// likelihood tolerances).  Per-point h (the adaptive search, whose
// Hooke-Jeeves steps compare nearby likelihoods): the FP64 exp.
template <bool VARH>
__device__ __forceinline__ double edge_factor(double d2, double h2, double k2) {
    if (VARH) return exp(d2 / (-2.0 * h2));
    const double a = d2 * k2;
    const float ah = (float)a;
    const float al = (float)(a - (double)ah);
    const float e = mgk_exp2_neg_poly(ah);
    return (double)__fmaf_rn(__fmul_rn(-al, MGK_LN2F), e, e);
}

// The oracle's FP64 cutoff decision for column c of a row at dy^2.
__device__ __forceinline__ bool in_cut(const mgk_grid& g, int64_t c, double px, double dy2, double cut) {
    const double dx = __dsub_rn(cell_xd(g, c), px);
    return __dadd_rn(__dmul_rn(dx, dx), dy2) < cut;
}

// Smallest c in [a, b] with in_cut true; in_cut is false..true over [a, b]
// and true at b.
__device__ __forceinline__ int64_t first_in(const mgk_grid& g, int64_t a, int64_t b, double px, double dy2,
                                            double cut) {
    while (a < b) {
        const int64_t m = a + ((b - a) >> 1);
        if (in_cut(g, m, px, dy2, cut)) b = m;
        else a = m + 1;
    }
    return a;
}

// Largest c in [a, b] with in_cut true; true..false over [a, b], true at a.
__device__ __forceinline__ int64_t last_in(const mgk_grid& g, int64_t a, int64_t b, double px, double dy2,
                                           double cut) {
    while (a < b) {
        const int64_t m = a + ((b - a + 1) >> 1);
        if (in_cut(g, m, px, dy2, cut)) a = m;
        else b = m - 1;
    }
    return a;
}

template <bool VARH>
__global__ void __launch_bounds__(kEdgeWarps * 32) k_edge_rows(EdgeParams E) {
    __shared__ double qsum[kEdgeWarps][kEdgeChunk + 1];
    const int lane = threadIdx.x & 31;
    double* Q = qsum[threadIdx.x >> 5];
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const mgk_grid g = E.g;
    const double xll = g.xll, yll = g.yll, cs = g.cs;
    const double inv_cs = 1.0 / cs;  // for the interval estimates, which the exact test then verifies
    const double cell_area = (double)(g.cs * g.cs);  // float product, kde_cuda_kdtr_tiled.cu:2698
    const int nh = VARH ? 1 : E.nh;
    unsigned long long cnt_total = 0;
    const int64_t ntask = E.list ? (int64_t)*E.list_count : E.n;
    for (int64_t t = warp0; t < ntask; t += nwarps) {
        const int64_t p = E.list ? (int64_t)E.list[t] : t;
        const double px = E.x[p], py = E.y[p];
        const double d2b = E.dist2 ? E.dist2[p] : 0.0;
        for (int k = 0; k < nh; k++) {
            const float hp = VARH ? E.hpp[p] : (E.hgrid ? E.hgrid[k] : E.hfix);
            const double h2 = mgk_h2(hp);
            const double cut = MGK_CUT * h2;
            float* out = E.ew + (int64_t)k * E.ew_stride + p;
            if (E.dist2 && d2b >= cut) {
                if (lane == 0) *out = 1.0f;
                continue;
            }
            const double reach = 3.0 * (double)hp;
            // NARROW window (kde_cuda_kdtr_tiled.cu:2719-2727), truncating casts as in Utilities.h:16-17
            int64_t rl = g.nrows - 1 - trunc_index((py + reach - yll) / cs);
            int64_t ru = g.nrows - 1 - trunc_index((py - reach - yll) / cs);
            int64_t cl = trunc_index((px - reach - xll) / cs);
            int64_t cu = trunc_index((px + reach - xll) / cs);
            rl = rl < 0 ? 0 : rl;
            ru = ru > g.nrows - 1 ? g.nrows - 1 : ru;
            cl = cl < 0 ? 0 : cl;
            cu = cu > g.ncols - 1 ? g.ncols - 1 : cu;
            const double k2 = MGK_LOG2E / (2.0 * h2);
            double acc = 0.0;
            unsigned long long cnt = 0;
            for (int64_t c0 = cl; c0 <= cu && rl <= ru; c0 += kEdgeChunk) {
                const int64_t c1 = mgk_min64(cu, c0 + kEdgeChunk - 1);
                const int len = (int)(c1 - c0 + 1);
                // prefix sums of the column factors: Q[j] = sum of the first j
                const int per = (len + 31) >> 5;
                const int j0 = min(len, lane * per), j1 = min(len, j0 + per);
                double run = 0.0;
                for (int j = j0; j < j1; j++) {
                    const double dx = __dsub_rn(cell_xd(g, c0 + j), px);
                    run += edge_factor<VARH>(__dmul_rn(dx, dx), h2, k2);
                    Q[j + 1] = run;
                }
                double off = run;
                for (int o = 1; o < 32; o <<= 1) {
                    const double v = __shfl_up_sync(0xffffffffu, off, o);
                    if (lane >= o) off += v;
                }
                off -= run;  // exclusive prefix of the segment totals
                for (int j = j0; j < j1; j++) Q[j + 1] += off;
                if (lane == 0) Q[0] = 0.0;
                __syncwarp();
                // the chunk column nearest the point: every non-empty row interval holds it
                int64_t a = c0, b = c1 + 1;
                while (a < b) {
                    const int64_t m = a + ((b - a) >> 1);
                    if (cell_xd(g, m) >= px) b = m;
                    else a = m + 1;
                }
                int64_t cm = a > c1 ? c1 : a;
                if (a > c0 && a <= c1 && __dsub_rn(px, cell_xd(g, a - 1)) < __dsub_rn(cell_xd(g, a), px)) cm = a - 1;
                for (int64_t r = rl + lane; r <= ru; r += 32) {
                    const double dy = __dsub_rn((double)mgk_cell_y(yll, cs, g.nrows, r), py);
                    const double dy2 = __dmul_rn(dy, dy);
                    if (dy2 >= cut || !in_cut(g, cm, px, dy2, cut)) continue;
                    const double t = sqrt(cut - dy2);
                    int64_t lo = clamp_index(ceil((px - t - xll) * inv_cs - 0.5), c0, cm);
                    if (in_cut(g, lo, px, dy2, cut)) {
                        if (lo > c0 && in_cut(g, lo - 1, px, dy2, cut)) lo = first_in(g, c0, lo - 1, px, dy2, cut);
                    } else {
                        lo = first_in(g, lo + 1, cm, px, dy2, cut);
                    }
                    int64_t hi = clamp_index(floor((px + t - xll) * inv_cs - 0.5), cm, c1);
                    if (in_cut(g, hi, px, dy2, cut)) {
                        if (hi < c1 && in_cut(g, hi + 1, px, dy2, cut)) hi = last_in(g, hi + 1, c1, px, dy2, cut);
                    } else {
                        hi = last_in(g, cm, hi - 1, px, dy2, cut);
                    }
                    // valid runs of the row clipped to [lo, hi]
                    int64_t q = E.run_start[r];
                    const int64_t qe = E.run_start[r + 1];
                    if (qe - q > 8) {  // first run ending after lo
                        int64_t x0 = q, x1 = qe;
                        while (x0 < x1) {
                            const int64_t m = x0 + ((x1 - x0) >> 1);
                            if (E.runs[m].y <= lo) x0 = m + 1;
                            else x1 = m;
                        }
                        q = x0;
                    }
                    double S = 0.0;
                    for (; q < qe; q++) {
                        const int2 rr = E.runs[q];
                        if (rr.y <= lo) continue;
                        if (rr.x > hi) break;
                        const int64_t ra = mgk_max64(rr.x, lo), rb = mgk_min64((int64_t)rr.y - 1, hi);
                        S += Q[rb - c0 + 1] - Q[ra - c0];
                        cnt += (unsigned long long)(rb - ra + 1);
                    }
                    if (S != 0.0) acc += edge_factor<VARH>(dy2, h2, k2) * S;
                }
                __syncwarp();
            }
            for (int o = 16; o; o >>= 1) {
                acc += __shfl_xor_sync(0xffffffffu, acc, o);
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            }
            if (lane == 0) {
                const double k0 = 1.0 / (h2 * (double)MGK_TWO_PI_F);
                *out = (float)(1.0 / (acc * k0 * cell_area));
                cnt_total += cnt;
            }
        }
    }
    if (E.evals && lane == 0 && cnt_total) atomicAdd(E.evals, cnt_total);
}

}  // namespace

int mgk_launch_edge_weights_multi(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* hpp,
                                  float hfix, const float* d_hgrid, int nh, const double* dist2,
                                  const mgk_raster* rc, float* ew_out, int64_t ew_stride,
                                  unsigned long long* d_evals) {
    if (n == 0 || nh <= 0) return MGK_OK;
    mgk_raster* r = const_cast<mgk_raster*>(rc);  // the run table is a cache of the mask
    int st;
    if ((st = mgk_raster_runs(ctx, r))) return st;
    EdgeParams E{};
    E.n = n;
    E.x = x;
    E.y = y;
    E.hpp = hpp;
    E.hgrid = d_hgrid;
    E.hfix = hfix;
    E.nh = hpp ? 1 : nh;
    E.dist2 = dist2;
    E.g = r->g;
    E.run_start = r->run_start;
    E.runs = r->runs;
    E.ew = ew_out;
    E.ew_stride = ew_stride;
    E.evals = d_evals;
    const int threads = kEdgeWarps * 32;
    // a grid-stride kernel: one resident wave, so that no CTA starts its
    // share only after the others have finished theirs
    int occ = 1;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, hpp ? (const void*)k_edge_rows<true> : (const void*)k_edge_rows<false>, threads, 0);
    if (e != cudaSuccess) return mgk_cuda_fail(ctx, e, "edge weights occupancy");
    occ = std::max(occ, 1);
    const int64_t blocks = std::min<int64_t>((int64_t)ctx->sm_count * occ, (n + kEdgeWarps - 1) / kEdgeWarps);
    int *list = nullptr, *count = nullptr;
    const size_t b_list = sizeof(int) * (size_t)n;
    const bool listed = E.nh == 1 && dist2 && n < (int64_t)INT32_MAX;
    if (listed) {
        if ((st = mgk_alloc(ctx, (void**)&list, b_list))) return st;
        if ((st = mgk_alloc(ctx, (void**)&count, sizeof(int)))) {
            mgk_free(ctx, list, b_list);
            return st;
        }
        e = cudaMemsetAsync(count, 0, sizeof(int), ctx->stream);
        if (e == cudaSuccess) {
            const unsigned gn = (unsigned)((n + 255) / 256);
            if (hpp) k_edge_near<true><<<gn, 256, 0, ctx->stream>>>(E, list, count);
            else k_edge_near<false><<<gn, 256, 0, ctx->stream>>>(E, list, count);
            e = cudaGetLastError();
        }
        E.list = list;
        E.list_count = count;
    }
    if (e == cudaSuccess) {
        if (hpp) k_edge_rows<true><<<(unsigned)blocks, threads, 0, ctx->stream>>>(E);
        else k_edge_rows<false><<<(unsigned)blocks, threads, 0, ctx->stream>>>(E);
        e = cudaGetLastError();
    }
    // back to the context's pool; later users are ordered after these kernels on the same stream
    if (listed) {
        mgk_free(ctx, list, b_list);
        mgk_free(ctx, count, sizeof(int));
    }
    if (e != cudaSuccess) return mgk_cuda_fail(ctx, e, "k_edge_rows");
    MGK_COUNT_LAUNCH(ctx, listed ? 2 : 1);
    return MGK_OK;
}

int mgk_launch_edge_weights(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* hpp, float h,
                            const double* dist2, const mgk_raster* r, float* ew_out,
                            unsigned long long* d_evals) {
    return mgk_launch_edge_weights_multi(ctx, n, x, y, hpp, h, nullptr, 1, dist2, r, ew_out, n, d_evals);
}
