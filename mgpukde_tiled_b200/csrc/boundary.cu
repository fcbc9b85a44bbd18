// Study-area boundary and point-to-boundary distances.
//
// dMarkBoundary (kde_kernel_kdtr.cu:1209-1281) marks a valid cell as boundary
// when it lies on the raster's outer ring or any of its 8 neighbours is NoData;
// MarkBoundary (kde_cuda_kdtr_tiled.cu:3956-4069) then keeps only those cells.
// dCalcDist2Boundary (kde_kernel_kdtr.cu:1285-1353) takes, per point, the
// minimum squared distance to every boundary-cell centre; the CPU twin
// (kde_cuda_kdtr_tiled.cu:4092-4133) keeps it in double, DBL_MAX when there is
// no boundary cell.  The distance gates the edge-correction short-circuit
// (weight 1 when dist2 >= 9 h^2), so it is computed exactly as the FP64 CPU
// path does: the minimum of exactly rounded double d^2 values.
//
// Here the mask is read once: the boundary test and the compaction of the
// boundary-cell centres happen in one pass.  The centres are then binned on a
// coarse grid (32 x 32 cells per bin) and each point searches rings of bins
// outward from its own, stopping once the nearest ring not yet searched
// cannot hold anything closer than the best distance found.  The minimum is
// order independent, so the result is the brute-force minimum bit for bit.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "mgk_internal.cuh"

namespace {

constexpr int kBinCells = 32;  // boundary bins are kBinCells x kBinCells mask cells

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

struct BinGrid {
    double x0, y0, side;  // lower-left corner of bin (0, 0), bin side in coordinates
    int nbx, nby;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ void bin_of(const BinGrid& B, double x, double y, int& bx, int& by) {
    const double fx = floor((x - B.x0) / B.side), fy = floor((y - B.y0) / B.side);
    bx = clampi((int)fmax(fmin(fx, 1e9), -1e9), 0, B.nbx - 1);
    by = clampi((int)fmax(fmin(fy, 1e9), -1e9), 0, B.nby - 1);
}

__global__ void k_bin_count(int64_t nb, const float2* __restrict__ cells, BinGrid B, int* __restrict__ cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nb) return;
    int bx, by;
    bin_of(B, cells[i].x, cells[i].y, bx, by);
    atomicAdd(&cnt[by * B.nbx + bx], 1);
}

// exclusive scan of n ints in one CTA (n is the boundary-bin count, small)
__global__ void __launch_bounds__(1024) k_scan_small(int* __restrict__ a, int n) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int chunk = (n + 1023) / 1024;
    const int b = t * chunk, e = min(n, b + chunk);
    int s = 0;
    for (int i = b; i < e; i++) s += a[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = t ? part[t - 1] : 0;
    for (int i = b; i < e; i++) {
        const int v = a[i];
        a[i] = run;
        run += v;
    }
    if (t == 1023) a[n] = part[1023];
}

__global__ void k_bin_fill(int64_t nb, const float2* __restrict__ cells, BinGrid B, const int* __restrict__ start,
                           int* __restrict__ cursor, float2* __restrict__ binned) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nb) return;
    int bx, by;
    bin_of(B, cells[i].x, cells[i].y, bx, by);
    const int k = by * B.nbx + bx;
    binned[start[k] + atomicAdd(&cursor[k], 1)] = cells[i];
}

__device__ __forceinline__ void scan_bin(const float2* __restrict__ cells, const int* __restrict__ start, int k,
                                         double px, double py, double& best) {
    for (int j = start[k]; j < start[k + 1]; j++) {
        const float2 c = cells[j];
        const double dx = __dsub_rn((double)c.x, px);
        const double dy = __dsub_rn((double)c.y, py);
        best = fmin(best, __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
    }
}

// Bin index of perimeter position i (0 <= i < 8r; i = 0 for r = 0) of the
// square ring r around (bx0, by0); false when that bin is off the grid.
__device__ __forceinline__ bool ring_bin(int r, int i, int bx0, int by0, const BinGrid& B, int& kk) {
    int bx, by;
    if (r == 0) {
        bx = bx0;
        by = by0;
    } else if (i < 2 * r + 1) {
        bx = bx0 - r + i;
        by = by0 - r;
    } else if (i < 4 * r + 2) {
        bx = bx0 - r + (i - 2 * r - 1);
        by = by0 + r;
    } else if (i < 6 * r + 1) {
        bx = bx0 - r;
        by = by0 - r + 1 + (i - 4 * r - 2);
    } else {
        bx = bx0 + r;
        by = by0 - r + 1 + (i - 6 * r - 1);
    }
    if (bx < 0 || by < 0 || bx >= B.nbx || by >= B.nby) return false;
    kk = by * B.nbx + bx;
    return true;
}

// Per bin: the smallest ring index (Chebyshev distance in bins) holding a
// non-empty bin; rings inside it are empty and are skipped by the search.
// One warp per bin, the lanes sharing each ring's perimeter.
__global__ void k_bin_near(const int* __restrict__ start, BinGrid B, int* __restrict__ near) {
    const int lane = threadIdx.x & 31;
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= B.nbx * B.nby) return;  // warp-uniform
    const int bx0 = k % B.nbx, by0 = k / B.nbx;
    const int rmax = max(B.nbx, B.nby);
    int found = rmax + 1;
    for (int r = 0; r <= rmax; r++) {
        const int per = r == 0 ? 1 : 8 * r;
        bool hit = false;
        for (int i = lane; i < per && !hit; i += 32) {
            int kk;
            hit = ring_bin(r, i, bx0, by0, B, kk) && start[kk + 1] > start[kk];
        }
        if (__any_sync(0xffffffffu, hit)) {
            found = r;
            break;
        }
    }
    if (lane == 0) near[k] = found;
}

__global__ void k_dist2_binned(int64_t n, const float* __restrict__ x, const float* __restrict__ y,
                               const float2* __restrict__ cells, const int* __restrict__ start,
                               const int* __restrict__ near, BinGrid B, double* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double px = x[i], py = y[i];
    int bx0, by0;
    bin_of(B, px, py, bx0, by0);
    double best = DBL_MAX;
    const int rmax = max(B.nbx, B.nby);
    for (int r = near[by0 * B.nbx + bx0]; r <= rmax; r++) {
        // ring r: bins at Chebyshev distance r from (bx0, by0)
        const int ylo = by0 - r, yhi = by0 + r, xlo = bx0 - r, xhi = bx0 + r;
        for (int bx = max(xlo, 0); bx <= min(xhi, B.nbx - 1); bx++) {
            if (ylo >= 0) scan_bin(cells, start, ylo * B.nbx + bx, px, py, best);
            if (r > 0 && yhi < B.nby) scan_bin(cells, start, yhi * B.nbx + bx, px, py, best);
        }
        for (int by = max(ylo + 1, 0); by <= min(yhi - 1, B.nby - 1); by++) {
            if (r > 0 && xlo >= 0) scan_bin(cells, start, by * B.nbx + xlo, px, py, best);
            if (r > 0 && xhi < B.nbx) scan_bin(cells, start, by * B.nbx + xhi, px, py, best);
        }
        // every bin beyond ring r is at least r full bins away from the point
        // (the margin covers rounding in the bin assignment)
        const double lb = (double)r * B.side * (1.0 - 1e-9);
        if (best <= lb * lb) break;
    }
    out[i] = best;
}

// ---- per-bin candidate lists ------------------------------------------------
// For a point p inside bin b (rectangle R), the nearest boundary cell c* obeys
// d(p, c*) <= UB_b = min_c maxdist(R, c) (the farthest corner of R from the
// best cell), so c* is among the cells with mindist(R, c) <= UB_b.  Each bin
// gets that candidate list once; its points then scan only the list.

__device__ __forceinline__ void bin_rect(const BinGrid& B, int bx, int by, double& x0, double& y0, double& x1,
                                         double& y1) {
    x0 = B.x0 + bx * B.side;
    y0 = B.y0 + by * B.side;
    x1 = x0 + B.side;
    y1 = y0 + B.side;
}

__device__ __forceinline__ double mind2(double x0, double y0, double x1, double y1, double cx, double cy) {
    const double dx = fmax(0.0, fmax(x0 - cx, cx - x1)), dy = fmax(0.0, fmax(y0 - cy, cy - y1));
    return dx * dx + dy * dy;
}

__device__ __forceinline__ double maxd2(double x0, double y0, double x1, double y1, double cx, double cy) {
    const double dx = fmax(fabs(cx - x0), fabs(cx - x1)), dy = fmax(fabs(cy - y0), fabs(cy - y1));
    return dx * dx + dy * dy;
}

// mode 0: UB per bin; mode 1: candidate count per bin; mode 2: fill the lists
// (one warp per bin; the lanes share each ring's perimeter bins)
// cap2: only cells within sqrt(cap2) of the bin rectangle are listed (points
// farther than that from every boundary cell get a distance above cap2).
template <int MODE>
__global__ void k_bin_cands(const float2* __restrict__ cells, const int* __restrict__ start,
                            const int* __restrict__ near, BinGrid B, double cap2, double* __restrict__ ub,
                            int* __restrict__ cnt, const int* __restrict__ cstart, float2* __restrict__ cand) {
    const int lane = threadIdx.x & 31;
    const int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (k >= B.nbx * B.nby) return;  // warp-uniform
    const int bx0 = k % B.nbx, by0 = k / B.nbx;
    double x0, y0, x1, y1;
    bin_rect(B, bx0, by0, x0, y0, x1, y1);
    const double widen = 1e-6 * B.side;
    x0 -= widen;
    y0 -= widen;
    x1 += widen;
    y1 += widen;
    const int rmax = max(B.nbx, B.nby);
    double lim = MODE == 0 ? cap2 : ub[k] * (1.0 + 1e-9);
    int n = 0;
    int base = MODE == 2 ? cstart[k] : 0;
    for (int r = near[k]; r <= rmax; r++) {
        const double lb = (double)(r > 0 ? r - 1 : 0) * B.side * (1.0 - 1e-9);
        if (lb * lb > lim) break;  // lim is warp-uniform
        const int per = r == 0 ? 1 : 8 * r;
        int mine = 0;
        for (int i = lane; i < per; i += 32) {
            int kk;
            if (!ring_bin(r, i, bx0, by0, B, kk)) continue;
            for (int j = start[kk]; j < start[kk + 1]; j++) {
                const double cx = cells[j].x, cy = cells[j].y;
                if (MODE == 0) lim = fmin(lim, maxd2(x0, y0, x1, y1, cx, cy));
                else if (mind2(x0, y0, x1, y1, cx, cy) <= lim) mine++;
            }
        }
        if (MODE == 0) {
            for (int o = 16; o; o >>= 1) lim = fmin(lim, __shfl_xor_sync(0xffffffffu, lim, o));
        } else {
            // lane offsets within the ring, then the matches are written in lane order
            int incl = mine;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            const int tot = __shfl_sync(0xffffffffu, incl, 31);
            if (MODE == 2 && mine) {
                int w = base + n + incl - mine;
                for (int i = lane; i < per; i += 32) {
                    int kk;
                    if (!ring_bin(r, i, bx0, by0, B, kk)) continue;
                    for (int j = start[kk]; j < start[kk + 1]; j++) {
                        const double cx = cells[j].x, cy = cells[j].y;
                        if (mind2(x0, y0, x1, y1, cx, cy) <= lim) cand[w++] = cells[j];
                    }
                }
            }
            n += tot;
        }
    }
    if (lane == 0) {
        if (MODE == 0) ub[k] = lim;
        if (MODE == 1) cnt[k] = n;
    }
}


// Points are searched in the order of their bins (a counting sort by bin),
// so the threads of a warp mostly walk one bin's candidate list: the list's
// loads are shared and the loop lengths agree.  Each result is stored by
// point index, so the order changes no value.
__global__ void k_point_bins(int64_t n, const float* __restrict__ x, const float* __restrict__ y, BinGrid B,
                             int* __restrict__ key, int* __restrict__ cnt) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int bx, by;
    bin_of(B, x[i], y[i], bx, by);
    key[i] = by * B.nbx + bx;
    atomicAdd(&cnt[key[i]], 1);
}

__global__ void k_point_order(int64_t n, const int* __restrict__ key, int* __restrict__ cursor,
                              int32_t* __restrict__ order) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    order[atomicAdd(&cursor[key[i]], 1)] = (int32_t)i;
}

__global__ void k_dist2_cands(int64_t n, const int32_t* __restrict__ order, const float* __restrict__ x,
                              const float* __restrict__ y, const float2* __restrict__ cells,
                              const int* __restrict__ start, const int* __restrict__ near,
                              const float2* __restrict__ cand, const int* __restrict__ cstart, BinGrid B,
                              double* __restrict__ out) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t i = order ? order[t] : t;
    const double px = x[i], py = y[i];
    double best = DBL_MAX;
    const double fx = floor((px - B.x0) / B.side), fy = floor((py - B.y0) / B.side);
    if (fx >= 0.0 && fy >= 0.0 && fx < (double)B.nbx && fy < (double)B.nby) {
        const int k = (int)fy * B.nbx + (int)fx;
        for (int j = cstart[k]; j < cstart[k + 1]; j++) {
            const float2 c = cand[j];
            const double dx = __dsub_rn((double)c.x, px);
            const double dy = __dsub_rn((double)c.y, py);
            best = fmin(best, __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        }
        out[i] = best;
        return;
    }
    // outside the bin grid: ring search from the nearest bin
    int bx0, by0;
    bin_of(B, px, py, bx0, by0);
    const int rmax = max(B.nbx, B.nby);
    for (int r = near[by0 * B.nbx + bx0]; r <= rmax; r++) {
        const int ylo = by0 - r, yhi = by0 + r, xlo = bx0 - r, xhi = bx0 + r;
        for (int bx = max(xlo, 0); bx <= min(xhi, B.nbx - 1); bx++) {
            if (ylo >= 0) scan_bin(cells, start, ylo * B.nbx + bx, px, py, best);
            if (r > 0 && yhi < B.nby) scan_bin(cells, start, yhi * B.nbx + bx, px, py, best);
        }
        for (int by = max(ylo + 1, 0); by <= min(yhi - 1, B.nby - 1); by++) {
            if (r > 0 && xlo >= 0) scan_bin(cells, start, by * B.nbx + xlo, px, py, best);
            if (r > 0 && xhi < B.nbx) scan_bin(cells, start, by * B.nbx + xhi, px, py, best);
        }
        const double lb = (double)r * B.side * (1.0 - 1e-9);
        if (best <= lb * lb) break;
    }
    out[i] = best;
}

// ---- valid-cell runs per row (used by the edge-correction integral) -------
// One warp per row: a run starts at a valid cell whose left neighbour is
// NoData (or the row's first cell) and ends after a valid cell whose right
// neighbour is NoData (or the row's last cell).  MODE 0 counts runs per row,
// MODE 1 writes them at the row's offset as half-open [a, b).
template <int MODE>
__global__ void k_row_runs(mgk_grid g, const float* __restrict__ mask, int64_t* __restrict__ start,
                           int2* __restrict__ runs) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (r >= g.nrows) return;  // warp-uniform
    const float* row = mask + r * g.ncols;
    const float nd = g.nodata;
    int64_t ns = 0, ne = 0;
    const int64_t base = MODE ? start[r] : 0;
    for (int64_t c0 = 0; c0 < g.ncols; c0 += 32) {
        const int64_t c = c0 + lane;
        bool v = false, vl = false, vr = false;
        if (c < g.ncols) {
            v = row[c] != nd;
            vl = c > 0 && row[c - 1] != nd;
            vr = c + 1 < g.ncols && row[c + 1] != nd;
        }
        const unsigned sm = __ballot_sync(0xffffffffu, v && !vl);
        const unsigned em = __ballot_sync(0xffffffffu, v && !vr);
        if (MODE) {
            const unsigned lt = (1u << lane) - 1u;
            if (v && !vl) runs[base + ns + __popc(sm & lt)].x = (int)c;
            if (v && !vr) runs[base + ne + __popc(em & lt)].y = (int)(c + 1);
        }
        ns += __popc(sm);
        ne += __popc(em);
    }
    if (!MODE && lane == 0) start[r] = ns;
}

// Exclusive scan of n int64 values in one CTA; the total goes to a[n].
__global__ void __launch_bounds__(1024) k_scan_i64(int64_t* __restrict__ a, int64_t n) {
    __shared__ int64_t part[1024];
    const int t = threadIdx.x;
    const int64_t chunk = (n + 1023) / 1024;
    const int64_t b = t * chunk, e = mgk_min64(n, b + chunk);
    int64_t s = 0;
    for (int64_t i = b; i < e; i++) s += a[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int64_t v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int64_t run = t ? part[t - 1] : 0;
    for (int64_t i = b; i < e; i++) {
        const int64_t v = a[i];
        a[i] = run;
        run += v;
    }
    if (t == 1023) a[n] = part[1023];
}

}  // namespace

int mgk_raster_runs(mgk_ctx* ctx, mgk_raster* r) {
    if (r->has_runs) return MGK_OK;
    const mgk_grid g = r->g;
    mgk_free(ctx, r->run_start, sizeof(int64_t) * (size_t)(g.nrows + 1));
    mgk_free(ctx, r->runs, sizeof(int2) * (size_t)std::max<int64_t>(r->nruns, 1));
    r->run_start = nullptr;
    r->runs = nullptr;
    r->nruns = 0;
    if (g.ncols > (int64_t)INT32_MAX - 1) return mgk_fail(ctx, MGK_ERR_INVALID, "raster wider than 2^31 - 2 columns");
    cudaStream_t s = ctx->stream;
    const size_t sb = sizeof(int64_t) * (size_t)(g.nrows + 1);
    int st;
    if ((st = mgk_alloc(ctx, (void**)&r->run_start, sb))) return st;
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(r->run_start, 0, sb, s));
    const unsigned grid = (unsigned)((g.nrows * 32 + 255) / 256);
    k_row_runs<0><<<grid, 256, 0, s>>>(g, r->mask, r->run_start, nullptr);
    k_scan_i64<<<1, 1024, 0, s>>>(r->run_start, g.nrows);
    MGK_CHECK_LAUNCH(ctx, "k_row_runs count");
    MGK_COUNT_LAUNCH(ctx, 2);
    int64_t total = 0;
    MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(&total, r->run_start + g.nrows, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    if ((st = mgk_alloc(ctx, (void**)&r->runs, sizeof(int2) * (size_t)std::max<int64_t>(total, 1)))) return st;
    r->nruns = total;
    k_row_runs<1><<<grid, 256, 0, s>>>(g, r->mask, r->run_start, r->runs);
    MGK_CHECK_LAUNCH(ctx, "k_row_runs fill");
    MGK_COUNT_LAUNCH(ctx, 1);
    r->has_runs = true;
    return MGK_OK;
}

int mgk_launch_mark_boundary(mgk_ctx* ctx, mgk_raster* r) {
    cudaStream_t s = ctx->stream;
    const mgk_grid g = r->g;
    const size_t ncell = (size_t)g.ncols * (size_t)g.nrows;
    int st;
    if (!r->boundary && (st = mgk_alloc(ctx, (void**)&r->boundary, ncell))) return st;
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
    if (r->bcells) mgk_free(ctx, r->bcells, sizeof(float2) * (size_t)std::max<int64_t>(r->nb, 1));
    if (r->bstart) mgk_free(ctx, r->bstart, sizeof(int) * (size_t)(r->nbins + 1));
    r->bcells = nullptr;
    r->bstart = nullptr;
    r->nb = (int64_t)nb;
    // bins of kBinCells x kBinCells mask cells over the mask extent
    r->bnx = (int)((g.ncols + kBinCells - 1) / kBinCells);
    r->bny = (int)((g.nrows + kBinCells - 1) / kBinCells);
    r->nbins = (int64_t)r->bnx * r->bny;
    const size_t b_cells = sizeof(float2) * (size_t)std::max<uint64_t>(nb, 1);
    const size_t b_start = sizeof(int) * (size_t)(r->nbins + 1);
    int* cursor = nullptr;
    if ((st = mgk_alloc(ctx, (void**)&r->bcells, b_cells)) || (st = mgk_alloc(ctx, (void**)&r->bstart, b_start)) ||
        (st = mgk_alloc(ctx, (void**)&cursor, b_start))) {
        mgk_free(ctx, cells, sizeof(float2) * ncell);
        return st;
    }
    BinGrid B{(double)g.xll, (double)g.yll, (double)kBinCells * (double)g.cs, r->bnx, r->bny};
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(r->bstart, 0, b_start, s));
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(cursor, 0, b_start, s));
    if (nb > 0) {
        const unsigned gb = (unsigned)((nb + 255) / 256);
        k_bin_count<<<gb, 256, 0, s>>>((int64_t)nb, cells, B, r->bstart);
        k_scan_small<<<1, 1024, 0, s>>>(r->bstart, (int)r->nbins);
        k_bin_fill<<<gb, 256, 0, s>>>((int64_t)nb, cells, B, r->bstart, cursor, r->bcells);
        MGK_CHECK_LAUNCH(ctx, "boundary bins");
        MGK_COUNT_LAUNCH(ctx, 3);
    }
    // cursor (nbins + 1 ints) is reused as the nearest-ring table
    k_bin_near<<<(unsigned)((r->nbins * 32 + 255) / 256), 256, 0, s>>>(r->bstart, B, cursor);
    MGK_CHECK_LAUNCH(ctx, "k_bin_near");
    MGK_COUNT_LAUNCH(ctx, 1);
    if (r->bnear) mgk_free(ctx, r->bnear, b_start);
    r->bnear = cursor;
    cursor = nullptr;
    // the per-bin candidate lists are built by the distance search, for its reach
    r->cand_cap = -1.0;
    MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    mgk_free(ctx, cells, sizeof(float2) * ncell);
    r->marked = true;
    // the mask may have changed since the runs were built
    r->has_runs = false;
    return mgk_raster_runs(ctx, r);
}

// Per-bin candidate lists for distances exact up to `cap` (coordinate units;
// infinite: every distance exact).  Bins whose nearest boundary cells lie
// beyond the cap get short or empty lists, so a small cap (3h: what the
// edge-weight short-circuit asks) makes the lists and the search cheap.
static int build_cands(mgk_ctx* ctx, mgk_raster* r, double cap) {
    cudaStream_t s = ctx->stream;
    const mgk_grid& g = r->g;
    BinGrid B{(double)g.xll, (double)g.yll, (double)kBinCells * (double)g.cs, r->bnx, r->bny};
    const size_t b_start = sizeof(int) * (size_t)(r->nbins + 1);
    const double cap2 = std::isfinite(cap) ? cap * cap * (1.0 + 1e-9) : DBL_MAX;
    if (r->bub) mgk_free(ctx, r->bub, sizeof(double) * (size_t)r->nbins);
    if (r->cstart) mgk_free(ctx, r->cstart, b_start);
    if (r->cand) mgk_free(ctx, r->cand, sizeof(float2) * (size_t)std::max<int64_t>(r->ncand, 1));
    r->bub = nullptr;
    r->cstart = nullptr;
    r->cand = nullptr;
    r->ncand = 0;
    r->cand_cap = -1.0;
    int st;
    if ((st = mgk_alloc(ctx, (void**)&r->bub, sizeof(double) * (size_t)r->nbins)) ||
        (st = mgk_alloc(ctx, (void**)&r->cstart, b_start)))
        return st;
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(r->cstart, 0, b_start, s));
    if (r->nb > 0) {
        const unsigned gbin = (unsigned)((r->nbins * 32 + 127) / 128);  // one warp per bin
        k_bin_cands<0><<<gbin, 128, 0, s>>>(r->bcells, r->bstart, r->bnear, B, cap2, r->bub, nullptr, nullptr, nullptr);
        k_bin_cands<1><<<gbin, 128, 0, s>>>(r->bcells, r->bstart, r->bnear, B, cap2, r->bub, r->cstart, nullptr, nullptr);
        k_scan_small<<<1, 1024, 0, s>>>(r->cstart, (int)r->nbins);
        MGK_CHECK_LAUNCH(ctx, "boundary candidate lists");
        MGK_COUNT_LAUNCH(ctx, 3);
        int total = 0;
        MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(&total, r->cstart + r->nbins, sizeof(int), cudaMemcpyDeviceToHost, s));
        MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
        r->ncand = total;
        if ((st = mgk_alloc(ctx, (void**)&r->cand, sizeof(float2) * (size_t)std::max(total, 1)))) return st;
        if (total > 0) {
            k_bin_cands<2><<<gbin, 128, 0, s>>>(r->bcells, r->bstart, r->bnear, B, cap2, r->bub, nullptr, r->cstart,
                                                r->cand);
            MGK_CHECK_LAUNCH(ctx, "boundary candidate fill");
            MGK_COUNT_LAUNCH(ctx, 1);
        }
    }
    r->cand_cap = std::isfinite(cap) ? cap : INFINITY;
    return MGK_OK;
}

int mgk_launch_dist2(mgk_ctx* ctx, mgk_points* p, mgk_raster* r, double cap) {
    if (!(r->cand_cap >= cap)) {  // no lists yet, or lists for a shorter reach
        int st = build_cands(ctx, r, cap);
        if (st) return st;
    }
    if (p->n == 0) return MGK_OK;
    const mgk_grid& g = r->g;
    BinGrid B{(double)g.xll, (double)g.yll, (double)kBinCells * (double)g.cs, r->bnx, r->bny};
    if (r->nb == 0) {
        k_dist2_binned<<<(unsigned)((p->n + 255) / 256), 256, 0, ctx->stream>>>(
            p->n, p->x, p->y, r->bcells, r->bstart, r->bnear, B, p->dist2);
    } else if (p->n >= (int64_t)INT32_MAX) {
        k_dist2_cands<<<(unsigned)((p->n + 255) / 256), 256, 0, ctx->stream>>>(
            p->n, nullptr, p->x, p->y, r->bcells, r->bstart, r->bnear, r->cand, r->cstart, B, p->dist2);
    } else {
        // counting sort of the points by bin, then the search in that order
        const size_t b_key = sizeof(int) * (size_t)p->n, b_cnt = sizeof(int) * (size_t)(r->nbins + 1);
        int *key = nullptr, *cnt = nullptr;
        int32_t* order = nullptr;
        int st;
        if ((st = mgk_alloc(ctx, (void**)&key, b_key))) return st;
        if ((st = mgk_alloc(ctx, (void**)&order, b_key)) || (st = mgk_alloc(ctx, (void**)&cnt, b_cnt))) {
            mgk_free(ctx, key, b_key);
            mgk_free(ctx, order, b_key);
            return st;
        }
        const unsigned gp = (unsigned)((p->n + 255) / 256);
        cudaError_t e = cudaMemsetAsync(cnt, 0, b_cnt, ctx->stream);
        if (e == cudaSuccess) {
            k_point_bins<<<gp, 256, 0, ctx->stream>>>(p->n, p->x, p->y, B, key, cnt);
            k_scan_small<<<1, 1024, 0, ctx->stream>>>(cnt, (int)r->nbins);
            k_point_order<<<gp, 256, 0, ctx->stream>>>(p->n, key, cnt, order);
            k_dist2_cands<<<gp, 256, 0, ctx->stream>>>(p->n, order, p->x, p->y, r->bcells, r->bstart, r->bnear,
                                                       r->cand, r->cstart, B, p->dist2);
            e = cudaGetLastError();
        }
        // the buffers go back to the context's pool; later users are ordered
        // after these kernels on the same stream
        mgk_free(ctx, key, b_key);
        mgk_free(ctx, order, b_key);
        mgk_free(ctx, cnt, b_cnt);
        if (e != cudaSuccess) return mgk_cuda_fail(ctx, e, "k_dist2");
        MGK_COUNT_LAUNCH(ctx, 3);
    }
    MGK_CHECK_LAUNCH(ctx, "k_dist2");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}
