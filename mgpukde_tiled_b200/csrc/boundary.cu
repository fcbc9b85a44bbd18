// Study-area boundary and point-to-boundary distances.
//
// dMarkBoundary (kde_kernel_kdtr.cu:1209-1281) marks a valid cell as boundary
// when it lies on the raster's outer ring or any of its 8 neighbours is NoData;
// MarkBoundary (kde_cuda_kdtr_tiled.cu:3956-4069) then keeps only those cells.
// dCalcDist2Boundary (kde_kernel_kdtr.cu:1285-1353) takes, per point, the
// minimum squared distance to every boundary-cell centre; the CPU twin
// (kde_cuda_kdtr_tiled.cu:4092-4133) keeps it in double, DBL_MAX when there is
// no boundary cell.  The distance only gates the edge-correction short-circuit
// (weight 1 when dist2 >= 9 h^2), so it is computed exactly as the FP64 CPU
// path does: the minimum of exactly rounded double d^2 values.
//
// Here the mask is read once: the boundary test and the compaction of the
// boundary-cell centres happen in one pass; the distance kernel streams the
// compacted centres through shared memory (one thread per point, FP64 math).
#include <cfloat>

#include "mgk_internal.cuh"

namespace {

__global__ void k_mark_boundary(mgk_grid g, const float* __restrict__ mask, uint8_t* __restrict__ out,
                                float2* __restrict__ cells, unsigned long long* __restrict__ count) {
    const int64_t ncell = g.ncols * g.nrows;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ncell;
         i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / g.ncols, c = i - r * g.ncols;
    const float nd = g.nodata;
    uint8_t b = 0;
    if (mask[i] != nd) {
        if (r == 0 || r == g.nrows - 1 || c == 0 || c == g.ncols - 1) {
            b = 1;
        } else {
            const float* up = mask + i - g.ncols;
            const float* dn = mask + i + g.ncols;
            b = (up[-1] == nd) | (up[0] == nd) | (up[1] == nd) | (mask[i - 1] == nd) | (mask[i + 1] == nd) |
                (dn[-1] == nd) | (dn[0] == nd) | (dn[1] == nd);
        }
    }
    out[i] = b;
    if (b) {
        const unsigned long long k = atomicAdd(count, 1ull);
        cells[k] = make_float2(mgk_cell_x(g.xll, g.cs, c), mgk_cell_y(g.yll, g.cs, g.nrows, r));
    }
    }
}

constexpr int kDistThreads = 256;
constexpr int kDistChunk = 2048;

__global__ void __launch_bounds__(kDistThreads) k_dist2(int64_t n, const float* __restrict__ x,
                                                        const float* __restrict__ y,
                                                        const float2* __restrict__ cells, int64_t nb,
                                                        double* __restrict__ out) {
    __shared__ float2 sc[kDistChunk];
    const int64_t i = blockIdx.x * (int64_t)kDistThreads + threadIdx.x;
    const bool live = i < n;
    const double px = live ? (double)x[i] : 0.0, py = live ? (double)y[i] : 0.0;
    double best = DBL_MAX;
    for (int64_t base = 0; base < nb; base += kDistChunk) {
        const int m = (int)mgk_min64(kDistChunk, nb - base);
        __syncthreads();
        for (int k = threadIdx.x; k < m; k += kDistThreads) sc[k] = cells[base + k];
        __syncthreads();
        if (live) {
#pragma unroll 4
            for (int k = 0; k < m; k++) {
                const float2 c = sc[k];
                const double dx = __dsub_rn((double)c.x, px);
                const double dy = __dsub_rn((double)c.y, py);
                const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
                best = fmin(best, d2);
            }
        }
    }
    if (live) out[i] = best;
}

}  // namespace

int mgk_launch_mark_boundary(mgk_ctx* ctx, mgk_raster* r) {
    cudaStream_t s = ctx->stream;
    const mgk_grid g = r->g;
    const size_t ncell = (size_t)g.ncols * (size_t)g.nrows;
    int st;
    if (!r->boundary && (st = mgk_alloc(ctx, (void**)&r->boundary, ncell))) return st;
    // Worst-case list size, trimmed after counting.
    float2* cells = nullptr;
    if ((st = mgk_alloc(ctx, (void**)&cells, sizeof(float2) * ncell))) return st;
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned long long), s));
    const unsigned grid = (unsigned)std::min<size_t>((ncell + 255) / 256, (size_t)ctx->sm_count * 32);
    k_mark_boundary<<<grid, 256, 0, s>>>(g, r->mask, r->boundary, cells, ctx->d_counter);
    MGK_CHECK_LAUNCH(ctx, "k_mark_boundary");
    MGK_COUNT_LAUNCH(ctx, 1);
    unsigned long long nb = 0;
    MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(&nb, ctx->d_counter, sizeof(nb), cudaMemcpyDeviceToHost, s));
    MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    if (r->bcells) mgk_free(ctx, r->bcells, sizeof(float2) * (size_t)r->nb);
    r->bcells = nullptr;
    r->nb = (int64_t)nb;
    if (nb > 0) {
        if ((st = mgk_alloc(ctx, (void**)&r->bcells, sizeof(float2) * nb))) {
            mgk_free(ctx, cells, sizeof(float2) * ncell);
            return st;
        }
        MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(r->bcells, cells, sizeof(float2) * nb, cudaMemcpyDeviceToDevice, s));
        MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    }
    mgk_free(ctx, cells, sizeof(float2) * ncell);
    r->marked = true;
    return MGK_OK;
}

int mgk_launch_dist2(mgk_ctx* ctx, mgk_points* p, const mgk_raster* r) {
    if (p->n == 0) return MGK_OK;
    k_dist2<<<(unsigned)((p->n + kDistThreads - 1) / kDistThreads), kDistThreads, 0, ctx->stream>>>(
        p->n, p->x, p->y, r->bcells, r->nb, p->dist2);
    MGK_CHECK_LAUNCH(ctx, "k_dist2");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}
