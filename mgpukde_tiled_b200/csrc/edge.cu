// Exact edge-correction weights (Diggle 1985).
//
// CalcEdgeCorrectionWeights (kde_kernel_kdtr.cu:117-189 fixed h, :192-265
// per-point h) and EdgeCorrectionWeightsExact (kde_cuda_kdtr_tiled.cu:2694-2807):
//   e_p = 1                                  if dist2_p >= 9 h^2
//   e_p = 1 / sum_{valid c, d^2 < 9h^2} K_h(d) cellArea   otherwise
// over the reference's NARROW row/column window (a superset of the 3h disc).
//
// One warp per point: rows of the window in turn, the 32 lanes across the
// row's columns, so each mask row segment is one coalesced read.  The cutoff
// is decided in FP64 exactly as the FP64 CPU path decides it; each in-cutoff
// term exp2(-dx^2 k2) * exp2(-dy^2 k2) is formed in FP32 from FP64 exponents
// (hi + lo split) and summed per lane with Kahan compensation; the lanes are
// merged in FP64 and the normalisation 1 / (sum * cellArea / (h^2 TWO_PI)) is
// taken in FP64.
#include <algorithm>

#include "mgk_internal.cuh"

namespace {

__device__ __forceinline__ int64_t trunc_index(double v) {
    v = fmin(fmax(v, -1.0e15), 1.0e15);
    return (int64_t)trunc(v);
}

constexpr int kEdgeThreads = 256;

__global__ void __launch_bounds__(kEdgeThreads) k_edge(int64_t n, const float* __restrict__ x,
                                                       const float* __restrict__ y,
                                                       const float* __restrict__ hpp, float hfix,
                                                       const double* __restrict__ dist2, mgk_grid g,
                                                       const float* __restrict__ mask, float* __restrict__ ew,
                                                       unsigned long long* __restrict__ evals) {
    const int lane = threadIdx.x & 31;
    const int64_t warp0 = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const double xll = g.xll, yll = g.yll, cs = g.cs;
    const double cell_area = (double)(g.cs * g.cs);  // float product, kde_cuda_kdtr_tiled.cu:2698
    unsigned long long cnt_total = 0;
    for (int64_t p = warp0; p < n; p += nwarps) {
        const float hp = hpp ? hpp[p] : hfix;
        const double h2 = mgk_h2(hp);
        const double cut = MGK_CUT * h2;
        if (dist2 && dist2[p] >= cut) {
            if (lane == 0) ew[p] = 1.0f;
            continue;
        }
        const float px = x[p], py = y[p];
        const double reach = 3.0 * (double)hp;
        // NARROW window (kde_cuda_kdtr_tiled.cu:2719-2727), truncating casts as in Utilities.h:16-17
        int64_t rl = g.nrows - 1 - trunc_index(((double)py + reach - yll) / cs);
        int64_t ru = g.nrows - 1 - trunc_index(((double)py - reach - yll) / cs);
        int64_t cl = trunc_index(((double)px - reach - xll) / cs);
        int64_t cu = trunc_index(((double)px + reach - xll) / cs);
        rl = rl < 0 ? 0 : rl;
        ru = ru > g.nrows - 1 ? g.nrows - 1 : ru;
        cl = cl < 0 ? 0 : cl;
        cu = cu > g.ncols - 1 ? g.ncols - 1 : cu;
        const double k2 = MGK_LOG2E / (2.0 * h2);
        float s = 0.0f, c = 0.0f;
        unsigned cnt = 0;
        for (int64_t r = rl; r <= ru; r++) {
            const float cy = mgk_cell_y(yll, cs, g.nrows, r);
            const double dy = __dsub_rn((double)cy, (double)py);
            const double dy2 = __dmul_rn(dy, dy);
            if (dy2 >= cut) continue;
            const float fy = mgk_exp2_neg(dy2 * k2);
            const float* mrow = mask + r * g.ncols;
            for (int64_t col = cl + lane; col <= cu; col += 32) {
                if (mrow[col] == g.nodata) continue;
                const float cx = mgk_cell_x(xll, cs, col);
                const double dx = __dsub_rn((double)cx, (double)px);
                const double dx2 = __dmul_rn(dx, dx);
                if (__dadd_rn(dx2, dy2) < cut) {
                    const float t = mgk_exp2_neg(dx2 * k2) * fy;
                    const float yk = t - c;
                    const float tk = s + yk;
                    c = (tk - s) - yk;
                    s = tk;
                    cnt++;
                }
            }
        }
        double v = (double)s - (double)c;
        for (int o = 16; o; o >>= 1) {
            v += __shfl_xor_sync(0xffffffffu, v, o);
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if (lane == 0) {
            const double k0 = 1.0 / (h2 * (double)MGK_TWO_PI_F);
            ew[p] = (float)(1.0 / (v * k0 * cell_area));
            cnt_total += cnt;
        }
    }
    if (evals && lane == 0 && cnt_total) atomicAdd(evals, cnt_total);
}

}  // namespace

int mgk_launch_edge_weights(mgk_ctx* ctx, int64_t n, const float* x, const float* y, const float* hpp, float h,
                            const double* dist2, const mgk_raster* r, float* ew_out,
                            unsigned long long* d_evals) {
    if (n == 0) return MGK_OK;
    const int64_t warps_needed = n;
    const int64_t max_blocks = (int64_t)ctx->sm_count * 16;
    const int64_t blocks = std::min<int64_t>(max_blocks, (warps_needed * 32 + kEdgeThreads - 1) / kEdgeThreads);
    k_edge<<<(unsigned)blocks, kEdgeThreads, 0, ctx->stream>>>(n, x, y, hpp, h, dist2, r->g, r->mask, ew_out,
                                                               d_evals);
    MGK_CHECK_LAUNCH(ctx, "k_edge");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}
