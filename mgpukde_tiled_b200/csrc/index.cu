// Cell-binned point index, built on the GPU.
//
// Replaces the reference's CPU k-d tree and its flattened GPU copy
// (KDtree.cu:53-154, CUDA_KDtree.cu:26-102) and the per-tile host halo filter
// (ExtractSamplePointsCurTile, kde_cuda_kdtr_tiled.cu:4672-4747).  Points are
// put into square bins of side `side` over their bounding box and stored
// bin-major, so the points of any run of bins along a bin row are one
// contiguous range: a raster tile's candidates within 3h are a handful of
// ranges, one per bin row.
//
// The sort is a stable LSD radix sort (8-bit digits) of the bin id, so the
// order inside a bin is the input order and every build is bitwise
// reproducible (the density sums are order-dependent in FP32).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "mgk_internal.cuh"

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 32;  // per thread per tile
constexpr int kSortTile = kSortThreads * kSortItems;

__device__ __forceinline__ unsigned f2ord(float f) {
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// bbox[0..3] = ordered-int min x, min y, max x, max y
__global__ void k_bbox(int64_t n, const float* __restrict__ x, const float* __restrict__ y,
                       unsigned* bbox) {
    unsigned mnx = 0xffffffffu, mny = 0xffffffffu, mxx = 0, mxy = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        unsigned ox = f2ord(x[i]), oy = f2ord(y[i]);
        mnx = min(mnx, ox);
        mny = min(mny, oy);
        mxx = max(mxx, ox);
        mxy = max(mxy, oy);
    }
    for (int o = 16; o; o >>= 1) {
        mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&bbox[0], mnx);
        atomicMin(&bbox[1], mny);
        atomicMax(&bbox[2], mxx);
        atomicMax(&bbox[3], mxy);
    }
}

__global__ void k_bin_keys(int64_t n, const float* __restrict__ x, const float* __restrict__ y,
                           double ox, double oy, double inv_side, int64_t nbx, int64_t nby,
                           unsigned* __restrict__ keys, int32_t* __restrict__ vals) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t bx = (int64_t)floor(((double)x[i] - ox) * inv_side);
    int64_t by = (int64_t)floor(((double)y[i] - oy) * inv_side);
    bx = bx < 0 ? 0 : (bx >= nbx ? nbx - 1 : bx);
    by = by < 0 ? 0 : (by >= nby ? nby - 1 : by);
    keys[i] = (unsigned)(by * nbx + bx);
    vals[i] = (int32_t)i;
}

// Per-tile histogram of one 8-bit digit: counts[d * ntiles + tile].
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(int64_t n, const unsigned* __restrict__ keys,
                                                             int shift, int ntiles, unsigned* __restrict__ counts) {
    __shared__ unsigned hist[256];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; k++) {
        int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&hist[(keys[i] >> shift) & 0xff], 1u);
    }
    __syncthreads();
    counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = hist[threadIdx.x];
}

// Exclusive scan of `len` counts in one CTA of 1024 threads (chunked).
__global__ void __launch_bounds__(1024) k_scan_exclusive(unsigned* __restrict__ data, int64_t len) {
    __shared__ unsigned long long part[1024];
    const int t = threadIdx.x;
    const int64_t chunk = (len + 1023) / 1024;
    const int64_t b = t * chunk, e = min(len, b + chunk);
    unsigned long long s = 0;
    for (int64_t i = b; i < e; i++) s += data[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        unsigned long long v = t >= off ? part[t - off] : 0ull;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned long long run = t ? part[t - 1] : 0ull;
    for (int64_t i = b; i < e; i++) {
        unsigned v = data[i];
        data[i] = (unsigned)run;
        run += v;
    }
}

// Stable scatter of one digit pass.  Items of a tile are taken in rounds of
// 256 (round-major, thread-minor = input order); inside a round the rank of an
// item among equal digits is its warp rank (match_any) plus the counts of the
// same digit in lower warps and in earlier rounds.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(
    int64_t n, const unsigned* __restrict__ keys_in, const int32_t* __restrict__ vals_in,
    unsigned* __restrict__ keys_out, int32_t* __restrict__ vals_out, int shift, int ntiles,
    const unsigned* __restrict__ offsets) {
    __shared__ unsigned warp_cnt[kSortThreads / 32][256];
    __shared__ unsigned warp_pre[kSortThreads / 32][256];
    __shared__ unsigned tile_base[256];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    tile_base[t] = offsets[(size_t)t * ntiles + blockIdx.x];
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; k++) {
        for (int w = 0; w < kSortThreads / 32; w++) warp_cnt[w][t] = 0;
        __syncthreads();
        const int64_t i = base + (int64_t)k * kSortThreads + t;
        const bool valid = i < n;
        unsigned key = 0, d = 0;
        int32_t val = 0;
        if (valid) {
            key = keys_in[i];
            val = vals_in[i];
            d = (key >> shift) & 0xff;
        }
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        unsigned rank = 0;
        if (valid) {
            const unsigned peers = __match_any_sync(vmask, d);
            rank = __popc(peers & ((1u << lane) - 1u));
            if (rank == 0) warp_cnt[wid][d] = __popc(peers);
        }
        __syncthreads();
        {
            unsigned run = 0;
            for (int w = 0; w < kSortThreads / 32; w++) {
                warp_pre[w][t] = run;
                run += warp_cnt[w][t];
            }
            warp_cnt[0][t] = run;  // round total for digit t (warp_cnt[0] reused)
        }
        __syncthreads();
        if (valid) {
            const unsigned pos = tile_base[d] + warp_pre[wid][d] + rank;
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncthreads();
        tile_base[t] += warp_cnt[0][t];
        __syncthreads();
    }
}

// bin_start[b] = first sorted position whose key >= b  (b in [0, nbins]).
__global__ void k_bin_starts(int64_t n, const unsigned* __restrict__ keys, int64_t nbins,
                             int32_t* __restrict__ start) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > n) return;
    const int64_t prev = i > 0 ? (int64_t)keys[i - 1] : -1;
    const int64_t cur = i < n ? (int64_t)keys[i] : nbins;
    for (int64_t b = prev + 1; b <= cur; b++) start[b] = (int32_t)i;
}

// A record's weight: w * e, divided by h^2 TWO_PI for per-point bandwidths
// (the per-point normalisation of the kernel).
__device__ __forceinline__ float record_wk(const float* __restrict__ w, const float* __restrict__ ew,
                                          const float* __restrict__ hpp, int32_t j) {
    float wk = (w ? w[j] : 1.0f) * (ew ? ew[j] : 1.0f);
    if (hpp) {
        const float hh = hpp[j] * hpp[j];
        wk = (float)((double)wk / ((double)hh * (double)MGK_TWO_PI_F));
    }
    return wk;
}

// The records' weights again, from the points' current edge weights.
__global__ void k_refresh_wk(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ w,
                             const float* __restrict__ ew, const float* __restrict__ hpp, MgkPt* __restrict__ out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i].wk = record_wk(w, ew, hpp, perm[i]);
}

__global__ void k_gather(int64_t n, const int32_t* __restrict__ perm, const float* __restrict__ x,
                         const float* __restrict__ y, const float* __restrict__ w,
                         const float* __restrict__ ew, const float* __restrict__ hpp, int qexp,
                         MgkPt* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t j = perm[i];
    MgkPt r;
    mgk_qsplit(x[j], qexp, r.xh, r.xl);
    mgk_qsplit(y[j], qexp, r.yh, r.yl);
    r.wk = record_wk(w, ew, hpp, j);
    r.k2h = r.k2l = r.hh = 0.0f;
    if (hpp) {
        const float hh = hpp[j] * hpp[j];
        const double h2 = (double)hh;
        const double k2 = MGK_LOG2E / (2.0 * h2);
        r.k2h = (float)k2;
        r.k2l = (float)(k2 - (double)r.k2h);
        r.hh = hh;
    }
    out[i] = r;
}

__global__ void k_hmax(int64_t n, const float* __restrict__ h, unsigned* out) {
    unsigned m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, f2ord(h[i]));
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Z-order (Morton) key of the bin of each index record: bit-interleaved bin
// column and row (16 bits each), value = the record's position.
__device__ __forceinline__ unsigned spread16(unsigned v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__global__ void k_morton_keys(int64_t n, const MgkPt* __restrict__ pts, double ox, double oy, double inv_side,
                              int64_t nbx, int64_t nby, unsigned* __restrict__ keys, int32_t* __restrict__ vals) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MgkPt p = pts[i];
    int64_t bx = (int64_t)floor(((double)(p.xh + p.xl) - ox) * inv_side);
    int64_t by = (int64_t)floor(((double)(p.yh + p.yl) - oy) * inv_side);
    bx = bx < 0 ? 0 : (bx >= nbx ? nbx - 1 : bx);
    by = by < 0 ? 0 : (by >= nby ? nby - 1 : by);
    keys[i] = spread16((unsigned)bx) | (spread16((unsigned)by) << 1);
    vals[i] = (int32_t)i;
}

// ---- halo selection: the points inside a rectangle, in input order -------
constexpr int kSelThreads = 256;
constexpr int kSelRounds = 16;
constexpr int kSelTile = kSelThreads * kSelRounds;

struct SelRect {
    double xlo, xhi, ylo, yhi;
};

__device__ __forceinline__ bool sel_in(const SelRect& R, float x, float y) {
    const double dx = (double)x, dy = (double)y;
    return dx >= R.xlo && dx <= R.xhi && dy >= R.ylo && dy <= R.yhi;
}

// Kept points per tile of kSelTile points; counts[ntiles] = 0 (the scan's total slot).
__global__ void __launch_bounds__(kSelThreads) k_sel_count(int64_t n, const float* __restrict__ x,
                                                           const float* __restrict__ y, SelRect R, int ntiles,
                                                           unsigned* __restrict__ counts) {
    __shared__ unsigned s_c;
    if (threadIdx.x == 0) s_c = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSelTile;
    unsigned c = 0;
    for (int r = 0; r < kSelRounds; r++) {
        const int64_t i = base + (int64_t)r * kSelThreads + threadIdx.x;
        c += (i < n && sel_in(R, x[i], y[i])) ? 1u : 0u;
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_c, c);
    __syncthreads();
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = s_c;
        if (blockIdx.x == 0) counts[ntiles] = 0;
    }
}

// Stable scatter: round-major, thread-minor order is the input order; the
// rank of a kept point is its warp ballot rank plus the kept points of lower
// warps in the round and of earlier rounds.
__global__ void __launch_bounds__(kSelThreads) k_sel_scatter(
    int64_t n, const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ w,
    const float* __restrict__ h, SelRect R, const unsigned* __restrict__ offsets, float* __restrict__ ox,
    float* __restrict__ oy, float* __restrict__ ow, float* __restrict__ oh) {
    __shared__ unsigned s_w[kSelThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kSelTile;
    unsigned run = offsets[blockIdx.x];
    for (int r = 0; r < kSelRounds; r++) {
        const int64_t i = base + (int64_t)r * kSelThreads + threadIdx.x;
        const bool keep = i < n && sel_in(R, x[i], y[i]);
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) s_w[warp] = __popc(bal);
        __syncthreads();
        unsigned before = 0, total = 0;
        for (int k = 0; k < kSelThreads / 32; k++) {
            before += k < warp ? s_w[k] : 0u;
            total += s_w[k];
        }
        if (keep) {
            const unsigned o = run + before + __popc(bal & ((1u << lane) - 1u));
            ox[o] = x[i];
            oy[o] = y[i];
            if (ow) ow[o] = w[i];
            if (oh) oh[o] = h[i];
        }
        run += total;
        __syncthreads();  // s_w is rewritten next round
    }
}

}  // namespace

// The points of src inside [xlo, xhi] x [ylo, yhi] (input order) into dst,
// whose arrays the caller allocates after the count: first call with dst ==
// NULL returns the count in *count (one read back), then with dst.
int mgk_launch_points_select(mgk_ctx* ctx, const mgk_points* src, double xlo, double xhi, double ylo, double yhi,
                             unsigned* d_scratch, int64_t* count, mgk_points* dst) {
    const int64_t n = src->n;
    const int ntiles = (int)((n + kSelTile - 1) / kSelTile);
    const SelRect R{xlo, xhi, ylo, yhi};
    cudaStream_t s = ctx->stream;
    if (!dst) {
        if (n == 0) {
            *count = 0;
            return MGK_OK;
        }
        k_sel_count<<<ntiles, kSelThreads, 0, s>>>(n, src->x, src->y, R, ntiles, d_scratch);
        k_scan_exclusive<<<1, 1024, 0, s>>>(d_scratch, ntiles + 1);
        MGK_CHECK_LAUNCH(ctx, "points select count");
        MGK_COUNT_LAUNCH(ctx, 2);
        unsigned tot = 0;
        MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(&tot, d_scratch + ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
        *count = (int64_t)tot;
        return MGK_OK;
    }
    if (n == 0 || dst->n == 0) return MGK_OK;
    k_sel_scatter<<<ntiles, kSelThreads, 0, s>>>(n, src->x, src->y, src->w, src->h, R, d_scratch, dst->x, dst->y,
                                                 src->w ? dst->w : nullptr, src->h ? dst->h : nullptr);
    MGK_CHECK_LAUNCH(ctx, "points select scatter");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}

int64_t mgk_points_select_scratch(int64_t n) { return (n + kSelTile - 1) / kSelTile + 1; }

// Positions of the index records in Z-order of their bins (stable: records
// of one bin keep their order).  Consecutive runs of this order are compact
// in both directions, unlike runs of the row-major record order.
int mgk_index_zorder(mgk_ctx* ctx, const mgk_index* idx, int32_t* d_order) {
    const int64_t n = idx->n;
    if (n == 0) return MGK_OK;
    if (idx->nbx > 65536 || idx->nby > 65536) return mgk_fail(ctx, MGK_ERR_INVALID, "index_zorder: bin grid too large");
    cudaStream_t s = ctx->stream;
    const int ntiles = (int)((n + kSortTile - 1) / kSortTile);
    const size_t b_keys = sizeof(unsigned) * (size_t)n, b_vals = sizeof(int32_t) * (size_t)n;
    const size_t b_cnt = sizeof(unsigned) * 256 * (size_t)ntiles;
    unsigned *k0 = nullptr, *k1 = nullptr, *cnt = nullptr;
    int32_t* v0 = nullptr;
    int st;
    if ((st = mgk_alloc(ctx, (void**)&k0, b_keys))) return st;
    if ((st = mgk_alloc(ctx, (void**)&k1, b_keys))) { mgk_free(ctx, k0, b_keys); return st; }
    if ((st = mgk_alloc(ctx, (void**)&v0, b_vals))) { mgk_free(ctx, k0, b_keys); mgk_free(ctx, k1, b_keys); return st; }
    if ((st = mgk_alloc(ctx, (void**)&cnt, b_cnt))) {
        mgk_free(ctx, k0, b_keys); mgk_free(ctx, k1, b_keys); mgk_free(ctx, v0, b_vals);
        return st;
    }
    k_morton_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, idx->pts, idx->ox, idx->oy, 1.0 / idx->side,
                                                             idx->nbx, idx->nby, k0, v0);
    const uint64_t maxb = (uint64_t)std::max(idx->nbx, idx->nby) - 1;
    int bits = 0;
    while (bits < 16 && (maxb >> bits) != 0) bits++;
    const int passes = std::max(1, (2 * bits + 7) / 8);
    unsigned *kin = k0, *kout = k1;
    int32_t *vin = v0, *vout = d_order;
    for (int p = 0; p < passes; p++) {
        k_radix_hist<<<ntiles, kSortThreads, 0, s>>>(n, kin, 8 * p, ntiles, cnt);
        k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, (int64_t)256 * ntiles);
        k_radix_scatter<<<ntiles, kSortThreads, 0, s>>>(n, kin, vin, kout, vout, 8 * p, ntiles, cnt);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && vin != d_order) e = cudaMemcpyAsync(d_order, vin, b_vals, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the scratch is released below
    MGK_COUNT_LAUNCH(ctx, 1 + 3 * passes);
    mgk_free(ctx, k0, b_keys);
    mgk_free(ctx, k1, b_keys);
    mgk_free(ctx, v0, b_vals);
    mgk_free(ctx, cnt, b_cnt);
    if (e != cudaSuccess) return mgk_cuda_fail(ctx, e, "index_zorder");
    return MGK_OK;
}

int mgk_index_refresh_weights(mgk_ctx* ctx, mgk_index* idx, const mgk_points* pts) {
    if (!idx || !pts || idx->n != pts->n) return mgk_fail(ctx, MGK_ERR_INVALID, "index_refresh_weights: bad arguments");
    if (idx->n == 0) return MGK_OK;
    k_refresh_wk<<<(unsigned)((idx->n + 255) / 256), 256, 0, ctx->stream>>>(
        idx->n, idx->perm, pts->w, pts->has_ew ? pts->ew : nullptr, idx->varh ? pts->h : nullptr, idx->pts);
    MGK_CHECK_LAUNCH(ctx, "k_refresh_wk");
    MGK_COUNT_LAUNCH(ctx, 1);
    return MGK_OK;
}

int mgk_launch_index_build(mgk_ctx* ctx, const mgk_points* pts, float h, float bin_size, mgk_index* idx) {
    const int64_t n = pts->n;
    cudaStream_t s = ctx->stream;
    idx->ctx = ctx;
    idx->n = n;
    idx->varh = (h <= 0.0f);
    if (idx->varh && !pts->h) return mgk_fail(ctx, MGK_ERR_INVALID, "index_build: h <= 0 but the points carry no per-point h");
    if (n >= (int64_t)INT32_MAX) return mgk_fail(ctx, MGK_ERR_INVALID, "index_build: too many points");
    // bounding box (and max h for per-point bandwidths) -> host
    unsigned* d_bb = reinterpret_cast<unsigned*>(ctx->d_counter);
    const unsigned init[6] = {0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u};
    MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(d_bb, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int red_blocks = std::max(1, std::min<int>(ctx->sm_count * 4, (int)((n + 255) / 256)));
    if (n > 0) {
        k_bbox<<<red_blocks, 256, 0, s>>>(n, pts->x, pts->y, d_bb);
        MGK_CHECK_LAUNCH(ctx, "k_bbox");
        if (idx->varh) {
            k_hmax<<<red_blocks, 256, 0, s>>>(n, pts->h, d_bb + 4);
            MGK_CHECK_LAUNCH(ctx, "k_hmax");
        }
    }
    unsigned hb[6];
    MGK_CHECK_CUDA(ctx, cudaMemcpyAsync(hb, d_bb, sizeof(hb), cudaMemcpyDeviceToHost, s));
    MGK_CHECK_CUDA(ctx, cudaStreamSynchronize(s));
    auto o2f = [](unsigned u) {
        unsigned v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
        float f;
        memcpy(&f, &v, 4);
        return f;
    };
    double xmin = 0, ymin = 0, xmax = 1, ymax = 1;
    if (n > 0) {
        xmin = o2f(hb[0]);
        ymin = o2f(hb[1]);
        xmax = o2f(hb[2]);
        ymax = o2f(hb[3]);
    }
    float hmax = h;
    if (idx->varh) hmax = n > 0 ? o2f(hb[4]) : 1.0f;
    if (!(hmax > 0.0f) || !std::isfinite(hmax)) return mgk_fail(ctx, MGK_ERR_INVALID, "index_build: bandwidths must be positive and finite");
    idx->h = idx->varh ? 0.0f : h;
    idx->h2 = mgk_h2(hmax);
    idx->cut_d2 = MGK_CUT * idx->h2;
    idx->k2 = MGK_LOG2E / (2.0 * idx->h2);
    idx->k0 = 1.0 / (idx->h2 * (double)MGK_TWO_PI_F);
    // 3h plus a margin: 9 h^2 is formed from the float square, which may
    // exceed h^2 by a relative 2^-24
    idx->reach = 3.0 * (double)hmax * (1.0 + 1e-6);
    double side = bin_size > 0.0f ? (double)bin_size : (double)ctx->bin_factor * (double)hmax;
    const double ext = std::max(xmax - xmin, ymax - ymin);
    side = std::max(side, ext / 4096.0);
    if (!(side > 0.0)) side = 1.0;
    idx->side = side;
    idx->ox = xmin;
    idx->oy = ymin;
    idx->nbx = (int64_t)std::floor((xmax - xmin) / side) + 1;
    idx->nby = (int64_t)std::floor((ymax - ymin) / side) + 1;
    const int64_t nbins = idx->nbx * idx->nby;
    // coordinate quantum: every coordinate within 3h (+ a bin) of a point is
    // below 2^(22 - qexp) in magnitude, so hi parts are exact floats and
    // differences of hi parts within the cutoff are exact
    const double maxabs = std::max(std::max(std::fabs(xmin), std::fabs(xmax)),
                                   std::max(std::fabs(ymin), std::fabs(ymax))) + 4.0 * idx->reach + 2.0 * side + 1.0;
    idx->qexp = 22 - (int)std::ceil(std::log2(maxabs));

    // allocations (persistent)
    const size_t b_start = sizeof(int32_t) * (size_t)(nbins + 1);
    const size_t b_pts = sizeof(MgkPt) * (size_t)std::max<int64_t>(n, 1);
    const size_t b_perm = sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1);
    int st;
    if ((st = mgk_alloc(ctx, (void**)&idx->bin_start, b_start))) return st;
    if ((st = mgk_alloc(ctx, (void**)&idx->pts, b_pts))) return st;
    if ((st = mgk_alloc(ctx, (void**)&idx->perm, b_perm))) return st;
    idx->bytes = b_start + b_pts + b_perm;

    // scratch: keys x2, vals x1 (+ perm as second value buffer), counts
    const int ntiles = (int)std::max<int64_t>(1, (n + kSortTile - 1) / kSortTile);
    const size_t b_keys = sizeof(unsigned) * (size_t)std::max<int64_t>(n, 1);
    const size_t b_vals = sizeof(int32_t) * (size_t)std::max<int64_t>(n, 1);
    const size_t b_cnt = sizeof(unsigned) * 256 * (size_t)ntiles;
    unsigned *k0 = nullptr, *k1 = nullptr, *cnt = nullptr;
    int32_t* v0 = nullptr;
    if ((st = mgk_alloc(ctx, (void**)&k0, b_keys))) return st;
    if ((st = mgk_alloc(ctx, (void**)&k1, b_keys))) { mgk_free(ctx, k0, b_keys); return st; }
    if ((st = mgk_alloc(ctx, (void**)&v0, b_vals))) { mgk_free(ctx, k0, b_keys); mgk_free(ctx, k1, b_keys); return st; }
    if ((st = mgk_alloc(ctx, (void**)&cnt, b_cnt))) {
        mgk_free(ctx, k0, b_keys); mgk_free(ctx, k1, b_keys); mgk_free(ctx, v0, b_vals);
        return st;
    }
    int rc = MGK_OK;
    do {
        if (n > 0) {
            k_bin_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, pts->x, pts->y, idx->ox, idx->oy,
                                                                   1.0 / side, idx->nbx, idx->nby, k0, v0);
            if ((rc = cudaGetLastError()) != cudaSuccess) { rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "k_bin_keys"); break; }
            int bits = 0;
            while (bits < 32 && ((uint64_t)(nbins - 1) >> bits) != 0) bits++;
            const int passes = std::max(1, (bits + 7) / 8);
            unsigned *kin = k0, *kout = k1;
            int32_t *vin = v0, *vout = idx->perm;
            for (int p = 0; p < passes; p++) {
                k_radix_hist<<<ntiles, kSortThreads, 0, s>>>(n, kin, 8 * p, ntiles, cnt);
                k_scan_exclusive<<<1, 1024, 0, s>>>(cnt, (int64_t)256 * ntiles);
                k_radix_scatter<<<ntiles, kSortThreads, 0, s>>>(n, kin, vin, kout, vout, 8 * p, ntiles, cnt);
                std::swap(kin, kout);
                std::swap(vin, vout);
            }
            if ((rc = cudaGetLastError()) != cudaSuccess) { rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "radix sort"); break; }
            // sorted keys in kin, values in vin; make sure perm holds the values
            if (vin != idx->perm) {
                if ((rc = cudaMemcpyAsync(idx->perm, vin, b_vals, cudaMemcpyDeviceToDevice, s)) != cudaSuccess) {
                    rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "perm copy");
                    break;
                }
            }
            k_bin_starts<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(n, kin, nbins, idx->bin_start);
            k_gather<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, idx->perm, pts->x, pts->y, pts->w,
                                                                 pts->has_ew ? pts->ew : nullptr,
                                                                 idx->varh ? pts->h : nullptr, idx->qexp, idx->pts);
            if ((rc = cudaGetLastError()) != cudaSuccess) { rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "index gather"); break; }
            MGK_COUNT_LAUNCH(ctx, (idx->varh ? 2 : 1) + 1 + 3 * passes + 2);
        } else {
            if ((rc = cudaMemsetAsync(idx->bin_start, 0, b_start, s)) != cudaSuccess) {
                rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "bin_start memset");
                break;
            }
        }
        // scratch must stay alive until the stream has used it
        if ((rc = cudaStreamSynchronize(s)) != cudaSuccess) { rc = mgk_cuda_fail(ctx, (cudaError_t)rc, "index build"); break; }
        rc = MGK_OK;
    } while (0);
    mgk_free(ctx, k0, b_keys);
    mgk_free(ctx, k1, b_keys);
    mgk_free(ctx, v0, b_vals);
    mgk_free(ctx, cnt, b_cnt);
    return rc;
}
