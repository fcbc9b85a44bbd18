// Leave-one-out log likelihood of a fixed bandwidth.
//
// LogLikelihood (kde_cuda_kdtr_tiled.cu:3214-3299) recomputes the edge
// weights at h, scatters K_h(d) w_i e_i into every neighbour of i found by a
// k-d tree range search (DensityAtPointsKdtr, kde_kernel_kdtr.cu:681-804),
// subtracts the self term and takes logf(max(den, EPSILONDENSITY))
// (dCopyDensityValues, :806-830), then sums in float (ReductionSum,
// :1045-1111).  Here the density at query point j is gathered directly over
// its neighbours i != j in the cell-binned index:
//   loo_j = sum_{i != j, d^2 < 9h^2} K_h(d) w_i e_i(h)
// one warp per query, the cutoff decided in FP64 exactly as the oracle does,
// terms in FP32 from FP64 exponents with Kahan compensation per lane, an FP64
// lane merge, log in FP64, and a fixed-order FP64 tree reduction over the
// queries (bitwise reproducible).
#include <algorithm>

#include "mgk_internal.cuh"

namespace {

constexpr int kLooThreads = 256;

__global__ void k_gather_ew(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ ew,
                            float* __restrict__ sew) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) sew[i] = ew ? ew[perm[i]] : 1.0f;
}

__global__ void __launch_bounds__(kLooThreads) k_loo(int64_t n, const MgkPt* __restrict__ pts,
                                                     const float* __restrict__ sew,
                                                     const int32_t* __restrict__ bin_start, double ox, double oy,
                                                     double inv_side, int64_t nbx, int64_t nby, float h,
                                                     double* __restrict__ logs,
                                                     unsigned long long* __restrict__ evals) {
    const int lane = threadIdx.x & 31;
    const int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (j >= n) return;
    const double h2 = mgk_h2(h);
    const double cut = MGK_CUT * h2;
    const double k2 = MGK_LOG2E / (2.0 * h2);
    const double reach = 3.0 * (double)h;
    const MgkPt qr = pts[j];
    const float2 q = make_float2(qr.xh + qr.xl, qr.yh + qr.yl);
    int64_t bx0 = (int64_t)floor(((double)q.x - reach - ox) * inv_side);
    int64_t bx1 = (int64_t)floor(((double)q.x + reach - ox) * inv_side);
    int64_t by0 = (int64_t)floor(((double)q.y - reach - oy) * inv_side);
    int64_t by1 = (int64_t)floor(((double)q.y + reach - oy) * inv_side);
    bx0 = mgk_max64(bx0, 0);
    by0 = mgk_max64(by0, 0);
    bx1 = mgk_min64(bx1, nbx - 1);
    by1 = mgk_min64(by1, nby - 1);
    float s = 0.0f, c = 0.0f;
    unsigned cnt = 0;
    for (int64_t by = by0; by <= by1; by++) {
        const int64_t sb = bin_start[by * nbx + bx0], se = bin_start[by * nbx + bx1 + 1];
        for (int64_t i = sb + lane; i < se; i += 32) {
            if (i == j) continue;
            const MgkPt p = pts[i];
            const double dx = __dsub_rn((double)(p.xh + p.xl), (double)q.x);
            const double dy = __dsub_rn((double)(p.yh + p.yl), (double)q.y);
            const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
            if (d2 < cut) {
                const float t = mgk_exp2_neg(d2 * k2) * (p.wk * sew[i]);
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
        const double loo = v / (h2 * (double)MGK_TWO_PI_F);
        const double floor_v = (double)MGK_EPS_DENSITY_F;
        logs[j] = log(loo > floor_v ? loo : floor_v);
        if (evals && cnt) atomicAdd(evals, (unsigned long long)cnt);
    }
}

// Fixed-order FP64 sum: each block sums a contiguous range with a tree, one
// partial per block; a second single-block pass sums the partials.
__global__ void k_sum_fixed(int64_t n, const double* __restrict__ in, double* __restrict__ out) {
    __shared__ double sh[256];
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b = blockIdx.x * per, e = mgk_min64(n, b + per);
    double v = 0.0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) v += in[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

}  // namespace

int mgk_launch_loo(mgk_ctx* ctx, const mgk_index* idx, const float* ew_input_order, float h, double* d_logl,
                   unsigned long long* d_evals) {
    const int64_t n = idx->n;
    cudaStream_t s = ctx->stream;
    if (n == 0) {
        MGK_CHECK_CUDA(ctx, cudaMemsetAsync(d_logl, 0, sizeof(double), s));
        return MGK_OK;
    }
    float* sew = nullptr;
    double* logs = nullptr;
    double* part = nullptr;
    const int nblk = 256;
    int st;
    if ((st = mgk_alloc(ctx, (void**)&sew, sizeof(float) * n))) return st;
    if ((st = mgk_alloc(ctx, (void**)&logs, sizeof(double) * n))) { mgk_free(ctx, sew, sizeof(float) * n); return st; }
    if ((st = mgk_alloc(ctx, (void**)&part, sizeof(double) * nblk))) {
        mgk_free(ctx, sew, sizeof(float) * n);
        mgk_free(ctx, logs, sizeof(double) * n);
        return st;
    }
    k_gather_ew<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, idx->perm, ew_input_order, sew);
    const int64_t blocks = (n * 32 + kLooThreads - 1) / kLooThreads;
    k_loo<<<(unsigned)blocks, kLooThreads, 0, s>>>(n, idx->pts, sew, idx->bin_start, idx->ox, idx->oy,
                                                   1.0 / idx->side, idx->nbx, idx->nby, h, logs, d_evals);
    k_sum_fixed<<<nblk, 256, 0, s>>>(n, logs, part);
    k_sum_fixed<<<1, 256, 0, s>>>(nblk, part, d_logl);
    cudaError_t ce = cudaGetLastError();
    MGK_COUNT_LAUNCH(ctx, 4);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    mgk_free(ctx, sew, sizeof(float) * n);
    mgk_free(ctx, logs, sizeof(double) * n);
    mgk_free(ctx, part, sizeof(double) * nblk);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "loo");
    return MGK_OK;
}
