// Density gather over the cell-binned index (one raster tile per call).
//
// Reference: KernelDesityEstimation_pPoints (kde_kernel_kdtr.cu:461-574) scatters
// each point's window into the tile with float atomicAdd, after
// InitCellDensities (:268-294) zeroed the valid cells.  Here every cell is
// owned by one thread that gathers:
//
//   den(c) = sum_p [d^2 < 9 h_p^2] exp(-d^2 / 2 h_p^2) / (h_p^2 TWO_PI) w_p e_p
//
// Layout: a CTA (256 threads) owns a 64 x 64 block of cells; warp w owns a
// 16 x 32 sub-block, lane l a 4 x 4 micro-tile.  The CTA stages the points of
// the bins within 3h of its block into shared memory, one contiguous range per
// bin row.  For each staged point a warp first tests its sub-block's
// rectangle against the 3h disc (exact, FP64) and skips the point if it
// cannot contribute.  Otherwise the Gaussian factorises over the grid:
//   exp2(-(a_j + b_i)) = E_j * F_i,  a_j = dx_j^2 k2, b_i = dy_i^2 k2,
//   k2 = log2(e) / (2 h^2)
// Each lane computes one column factor E (32 columns) and one row factor F
// (16 rows) with an FP64 exponent split into float hi+lo, the warp exchanges
// them through shared memory, and each lane forms its 16 products with one
// FMUL each.  The cutoff d^2 < 9h^2 is decided in FP32 as a_j < cut - b_i;
// pairs within a narrow band of the cutoff (|a_j + b_i - cut| < 4e-6, log2
// units) are re-decided with the exact FP64 test the oracle uses, so the set
// of summed pairs equals the reference's.
//
// Accumulation: per cell, FP32 partial sums over 8 points are added into a
// Kahan-compensated FP32 accumulator; the result is formed in FP64
// (sum - compensation) times the kernel normalisation.  Blocks with many
// candidates are split across CTAs (work items); their partial sums are
// written in FP64 to scratch and merged in a fixed order, so results are
// bitwise reproducible.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mgk_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kBlk = 64;       // cells per CTA block side
constexpr int kChunk = 512;    // points staged per batch
constexpr float kAmbEps = 4e-6f;

struct Item {
    int32_t bx, by;       // block coordinates within the tile
    int32_t k0, k1;       // candidate range in the block's candidate sequence
    int32_t slot;         // scratch slot (split blocks) or -1 (direct store)
    int32_t pad;
};

struct DParams {
    double xll, yll, cs;
    int64_t g_nrows;
    int64_t row0, col0, nr, nc;
    float nodata;
    const float* mask;
    float* out;
    double* scratch;  // [slot][kBlk*kBlk]
    const Item* items;
    // index
    const float4* pts;
    const double2* hk;
    const int32_t* bin_start;
    double ox, oy, inv_side;
    int64_t nbx, nby;
    // fixed-h constants
    double h2, k2, k0, cut_d2, cutl, reach;
    unsigned long long* evals;
};

// Bin range covering [lo, hi] (coordinates), clamped; returns false if empty.
__device__ __forceinline__ bool bin_range(double lo, double hi, double o, double inv_side, int64_t nb,
                                          int64_t& a, int64_t& b) {
    double fa = floor((lo - o) * inv_side), fb = floor((hi - o) * inv_side);
    if (fb < 0.0 || fa > (double)(nb - 1)) return false;
    a = fa < 0.0 ? 0 : (int64_t)fa;
    b = fb > (double)(nb - 1) ? nb - 1 : (int64_t)fb;
    return true;
}

struct BlockGeom {
    int64_t r0, c0;   // global first row / col of the block
    int nrow, ncol;   // cells of the block inside the tile
    int64_t bx0, bx1, by0, by1;
    bool any;
};

__device__ __forceinline__ BlockGeom block_geom(const DParams& P, int bxi, int byi) {
    BlockGeom G;
    G.r0 = P.row0 + (int64_t)byi * kBlk;
    G.c0 = P.col0 + (int64_t)bxi * kBlk;
    G.nrow = (int)mgk_min64(kBlk, P.row0 + P.nr - G.r0);
    G.ncol = (int)mgk_min64(kBlk, P.col0 + P.nc - G.c0);
    const double x_lo = mgk_cell_x(P.xll, P.cs, G.c0), x_hi = mgk_cell_x(P.xll, P.cs, G.c0 + G.ncol - 1);
    const double y_hi = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0);
    const double y_lo = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + G.nrow - 1);
    G.any = bin_range(x_lo - P.reach, x_hi + P.reach, P.ox, P.inv_side, P.nbx, G.bx0, G.bx1) &&
            bin_range(y_lo - P.reach, y_hi + P.reach, P.oy, P.inv_side, P.nby, G.by0, G.by1);
    return G;
}

// Candidate count of every block of the tile (planning).
__global__ void k_block_counts(DParams P, int nbx_t, int nby_t, int64_t* __restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nbx_t * nby_t) return;
    const BlockGeom G = block_geom(P, i % nbx_t, i / nbx_t);
    int64_t c = 0;
    if (G.any)
        for (int64_t by = G.by0; by <= G.by1; by++)
            c += (int64_t)P.bin_start[by * P.nbx + G.bx1 + 1] - (int64_t)P.bin_start[by * P.nbx + G.bx0];
    counts[i] = c;
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

template <bool VARH, bool COUNT>
__global__ void __launch_bounds__(kThreads, 2) k_density(DParams P) {
    __shared__ float4 sp[kChunk];
    __shared__ double2 shk[VARH ? kChunk : 1];
    __shared__ double scx[kBlk], scy[kBlk];
    __shared__ float2 colbuf[kThreads / 32][2][32];
    __shared__ float2 rowbuf[kThreads / 32][2][16];

    const Item it = P.items[blockIdx.x];
    const BlockGeom G = block_geom(P, it.bx, it.by);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp >> 1, wc = warp & 1;      // warp sub-block: rows wr*16.., cols wc*32..
    const int tr = lane >> 3, tc = lane & 7;      // lane micro-tile: rows tr*4.., cols tc*4..
    if (tid < kBlk) scx[tid] = (double)mgk_cell_x(P.xll, P.cs, G.c0 + tid);
    else if (tid < 2 * kBlk) scy[tid - kBlk] = (double)mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + tid - kBlk);
    __syncthreads();

    const bool warp_on = (wr * 16 < G.nrow) && (wc * 32 < G.ncol);
    // warp rectangle (cell centres), clamped to cells inside the tile
    const double wx0 = scx[wc * 32], wx1 = scx[min(wc * 32 + 31, G.ncol - 1)];
    const double wy1 = scy[wr * 16], wy0 = scy[min(wr * 16 + 15, G.nrow - 1)];
    const double my_cx = scx[wc * 32 + lane];
    const double my_cy = scy[wr * 16 + (lane & 15)];

    // validity of the lane's 16 cells (inside the tile and not NoData)
    unsigned valid = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = wr * 16 + tr * 4 + i, c = wc * 32 + tc * 4 + j;
            bool v = r < G.nrow && c < G.ncol;
            if (v && P.mask) v = P.mask[(G.r0 + r - P.row0) * P.nc + (G.c0 + c - P.col0)] != P.nodata;
            valid |= (unsigned)v << (i * 4 + j);
        }

    float acc_s[16], acc_c[16], part[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc_s[k] = acc_c[k] = part[k] = 0.0f;
    unsigned long long cnt = 0;
    unsigned pc = 0;  // points processed by this warp (warp-uniform)

    if (G.any) {
        int64_t seq = 0;  // position in the block's candidate sequence
        for (int64_t by = G.by0; by <= G.by1 && seq < it.k1; by++) {
            const int64_t sb = P.bin_start[by * P.nbx + G.bx0];
            const int64_t se = P.bin_start[by * P.nbx + G.bx1 + 1];
            const int64_t len = se - sb;
            // intersect [seq, seq+len) with [k0, k1)
            const int64_t lo = mgk_max64(seq, it.k0), hi = mgk_min64(seq + len, it.k1);
            for (int64_t base = lo; base < hi; base += kChunk) {
                const int m = (int)mgk_min64(kChunk, hi - base);
                const int64_t src = sb + (base - seq);
                __syncthreads();
                for (int k = tid; k < m; k += kThreads) {
                    sp[k] = P.pts[src + k];
                    if (VARH) shk[k] = P.hk[src + k];
                }
                __syncthreads();
                if (!warp_on) continue;
                for (int q = 0; q < m; q++) {
                    const float4 p = sp[q];
                    double h2, k2, cut_d2;
                    if (VARH) {
                        const double2 hk = shk[q];
                        h2 = hk.x;
                        k2 = hk.y;
                        cut_d2 = MGK_CUT * h2;
                    } else {
                        h2 = P.h2;
                        k2 = P.k2;
                        cut_d2 = P.cut_d2;
                    }
                    (void)h2;
                    // exact rectangle test: skip if no cell centre of the sub-block is within 3h
                    {
                        const double px = p.x, py = p.y;
                        const double ddx = fmax(0.0, fmax(__dsub_rn(wx0, px), __dsub_rn(px, wx1)));
                        const double ddy = fmax(0.0, fmax(__dsub_rn(wy0, py), __dsub_rn(py, wy1)));
                        if (__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)) >= cut_d2) continue;
                    }
                    const int b = pc & 1;
                    {
                        const double dx = (double)p.x - my_cx;
                        const double a = dx * dx * k2;
                        colbuf[warp][b][lane] = make_float2(__double2float_rn(a), mgk_exp2_neg(a));
                    }
                    if (lane < 16) {
                        const double dy = (double)p.y - my_cy;
                        const double bb = dy * dy * k2;
                        const double cutl = VARH ? MGK_CUT * 0.5 * MGK_LOG2E : P.cutl;
                        rowbuf[warp][b][lane] = make_float2(__double2float_rn(cutl - bb), p.z * mgk_exp2_neg(bb));
                    }
                    __syncwarp();
                    float ca[4], ce[4], rt[4], re[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        const float2 v = colbuf[warp][b][tc * 4 + j];
                        ca[j] = v.x;
                        ce[j] = v.y;
                    }
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const float2 v = rowbuf[warp][b][tr * 4 + i];
                        rt[i] = v.x;
                        re[i] = v.y;
                    }
                    bool amb = false;
                    unsigned inm = 0;
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const float u = ca[j] - rt[i];
                            const bool in = u < 0.0f;
                            amb |= fabsf(u) < kAmbEps;
                            if (in) part[i * 4 + j] += ce[j] * re[i];
                            if (COUNT) inm |= (unsigned)in << (i * 4 + j);
                        }
                    if (__any_sync(0xffffffffu, amb)) {
                        if (amb) {
#pragma unroll
                            for (int i = 0; i < 4; i++)
#pragma unroll
                                for (int j = 0; j < 4; j++) {
                                    const float u = ca[j] - rt[i];
                                    if (fabsf(u) < kAmbEps) {
                                        const float cxf = (float)scx[wc * 32 + tc * 4 + j];
                                        const float cyf = (float)scy[wr * 16 + tr * 4 + i];
                                        const bool ex = mgk_d2_exact(p.x, p.y, cxf, cyf) < cut_d2;
                                        const bool fl = u < 0.0f;
                                        if (ex != fl) {
                                            const float t = ce[j] * re[i];
                                            part[i * 4 + j] += ex ? t : -t;
                                            if (COUNT) inm ^= 1u << (i * 4 + j);
                                        }
                                    }
                                }
                        }
                    }
                    if (COUNT) cnt += __popc(inm & valid);
                    pc++;
                    if ((pc & 7u) == 0) {
#pragma unroll
                        for (int k = 0; k < 16; k++) {
                            kahan_add(acc_s[k], acc_c[k], part[k]);
                            part[k] = 0.0f;
                        }
                    }
                }
            }
            seq += len;
        }
    }
#pragma unroll
    for (int k = 0; k < 16; k++) kahan_add(acc_s[k], acc_c[k], part[k]);

    // epilogue: FP64 result = (s - c) * normalisation
    const double norm = VARH ? 1.0 : P.k0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int k = i * 4 + j;
            const int r = wr * 16 + tr * 4 + i, c = wc * 32 + tc * 4 + j;
            if (r >= G.nrow || c >= G.ncol) continue;
            const double v = ((double)acc_s[k] - (double)acc_c[k]) * norm;
            if (it.slot >= 0) {
                P.scratch[(size_t)it.slot * (kBlk * kBlk) + r * kBlk + c] = v;
            } else {
                const int64_t o = (G.r0 + r - P.row0) * P.nc + (G.c0 + c - P.col0);
                P.out[o] = ((valid >> k) & 1u) ? (float)v : P.nodata;
            }
        }
    if (COUNT) {
        for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0 && cnt) atomicAdd(P.evals, cnt);
    }
}

// Plain FP64 form: same blocks, staging and candidate lists; per pair an
// exact FP64 distance, the cutoff, a double exp and a double accumulate.
template <bool VARH>
__global__ void __launch_bounds__(kThreads, 2) k_density_fp64(DParams P) {
    __shared__ float4 sp[kChunk];
    __shared__ double2 shk[VARH ? kChunk : 1];
    const Item it = P.items[blockIdx.x];
    const BlockGeom G = block_geom(P, it.bx, it.by);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = warp >> 1, wc = warp & 1, tr = lane >> 3, tc = lane & 7;
    float cx[4], cy[4];
#pragma unroll
    for (int j = 0; j < 4; j++) cx[j] = mgk_cell_x(P.xll, P.cs, G.c0 + wc * 32 + tc * 4 + j);
#pragma unroll
    for (int i = 0; i < 4; i++) cy[i] = mgk_cell_y(P.yll, P.cs, P.g_nrows, G.r0 + wr * 16 + tr * 4 + i);
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; k++) acc[k] = 0.0;
    unsigned long long cnt = 0;
    if (G.any) {
        int64_t seq = 0;
        for (int64_t by = G.by0; by <= G.by1 && seq < it.k1; by++) {
            const int64_t sb = P.bin_start[by * P.nbx + G.bx0];
            const int64_t se = P.bin_start[by * P.nbx + G.bx1 + 1];
            const int64_t len = se - sb;
            const int64_t lo = mgk_max64(seq, it.k0), hi = mgk_min64(seq + len, it.k1);
            for (int64_t base = lo; base < hi; base += kChunk) {
                const int m = (int)mgk_min64(kChunk, hi - base);
                const int64_t src = sb + (base - seq);
                __syncthreads();
                for (int k = tid; k < m; k += kThreads) {
                    sp[k] = P.pts[src + k];
                    if (VARH) shk[k] = P.hk[src + k];
                }
                __syncthreads();
                for (int q = 0; q < m; q++) {
                    const float4 p = sp[q];
                    const double h2 = VARH ? shk[q].x : P.h2;
                    const double cut = MGK_CUT * h2;
                    const double m2h = -1.0 / (2.0 * h2);
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const double d2 = mgk_d2_exact(p.x, p.y, cx[j], cy[i]);
                            if (d2 < cut) {
                                acc[i * 4 + j] += exp(d2 * m2h) * (double)p.z;
                                cnt++;
                            }
                        }
                }
            }
            seq += len;
        }
    }
    const double norm = VARH ? 1.0 : P.k0;
    unsigned long long vcnt = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int r = wr * 16 + tr * 4 + i, c = wc * 32 + tc * 4 + j;
            if (r >= G.nrow || c >= G.ncol) continue;
            const double v = acc[i * 4 + j] * norm;
            if (it.slot >= 0) {
                P.scratch[(size_t)it.slot * (kBlk * kBlk) + r * kBlk + c] = v;
            } else {
                const int64_t o = (G.r0 + r - P.row0) * P.nc + (G.c0 + c - P.col0);
                const bool valid = !P.mask || P.mask[o] != P.nodata;
                P.out[o] = valid ? (float)v : P.nodata;
            }
        }
    (void)vcnt;
    (void)cnt;
}

// Merge of split blocks: cell value = sum over the block's slots in order.
__global__ void k_merge(DParams P, const int32_t* __restrict__ blocks, const int32_t* __restrict__ slot_begin,
                        int nbx_t) {
    const int b = blockIdx.x;
    const int32_t blk = blocks[b];
    const int s0 = slot_begin[b], s1 = slot_begin[b + 1];
    const int bxi = blk % nbx_t, byi = blk / nbx_t;
    const int64_t r0 = P.row0 + (int64_t)byi * kBlk, c0 = P.col0 + (int64_t)bxi * kBlk;
    const int nrow = (int)mgk_min64(kBlk, P.row0 + P.nr - r0);
    const int ncol = (int)mgk_min64(kBlk, P.col0 + P.nc - c0);
    for (int e = threadIdx.x; e < kBlk * kBlk; e += blockDim.x) {
        const int r = e / kBlk, c = e % kBlk;
        if (r >= nrow || c >= ncol) continue;
        double v = 0.0;
        for (int s = s0; s < s1; s++) v += P.scratch[(size_t)s * (kBlk * kBlk) + e];
        const int64_t o = (r0 + r - P.row0) * P.nc + (c0 + c - P.col0);
        const bool valid = !P.mask || P.mask[o] != P.nodata;
        P.out[o] = valid ? (float)v : P.nodata;
    }
}

}  // namespace

int mgk_launch_density(mgk_ctx* ctx, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                       int64_t nr, int64_t nc, const float* d_mask, float* d_out,
                       unsigned long long* d_evals, bool fp64) {
    if (nr <= 0 || nc <= 0) return MGK_OK;
    cudaStream_t s = ctx->stream;
    DParams P{};
    P.xll = g->xll;
    P.yll = g->yll;
    P.cs = g->cs;
    P.g_nrows = g->nrows;
    P.row0 = row0;
    P.col0 = col0;
    P.nr = nr;
    P.nc = nc;
    P.nodata = g->nodata;
    P.mask = d_mask;
    P.out = d_out;
    P.pts = idx->pts;
    P.hk = idx->hk;
    P.bin_start = idx->bin_start;
    P.ox = idx->ox;
    P.oy = idx->oy;
    P.inv_side = 1.0 / idx->side;
    P.nbx = idx->nbx;
    P.nby = idx->nby;
    P.h2 = idx->h2;
    P.k2 = idx->k2;
    P.k0 = idx->k0;
    P.cut_d2 = idx->cut_d2;
    P.cutl = idx->cut_d2 * idx->k2;
    P.reach = idx->reach;
    P.evals = d_evals;

    const int nbx_t = (int)((nc + kBlk - 1) / kBlk), nby_t = (int)((nr + kBlk - 1) / kBlk);
    const int nblk = nbx_t * nby_t;
    int st;
    // ---- plan: candidates per block -> work items (split heavy blocks) ----
    int64_t* d_counts = nullptr;
    if ((st = mgk_alloc(ctx, (void**)&d_counts, sizeof(int64_t) * nblk))) return st;
    k_block_counts<<<(nblk + 255) / 256, 256, 0, s>>>(P, nbx_t, nby_t, d_counts);
    std::vector<int64_t> counts(nblk);
    cudaError_t ce = cudaMemcpyAsync(counts.data(), d_counts, sizeof(int64_t) * nblk, cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    mgk_free(ctx, d_counts, sizeof(int64_t) * nblk);
    if (ce != cudaSuccess) return mgk_cuda_fail(ctx, ce, "density plan");

    int64_t total = 0, maxc = 0;
    for (int64_t c : counts) {
        total += c;
        maxc = std::max(maxc, c);
    }
    // Items of at most K candidates: about 8 waves of the resident CTAs.
    const int64_t slots_resident = (int64_t)ctx->sm_count * 2;
    int64_t K = std::max<int64_t>(2048, total / std::max<int64_t>(1, slots_resident * 8));
    K = (K + kChunk - 1) / kChunk * kChunk;
    std::vector<Item> items;
    std::vector<int32_t> split_blocks, split_begin;
    int32_t nslots = 0;
    items.reserve(nblk + 16);
    for (int b = 0; b < nblk; b++) {
        const int64_t c = counts[b];
        const int bxi = b % nbx_t, byi = b / nbx_t;
        if (c <= K) {
            items.push_back({bxi, byi, 0, (int32_t)c, -1, 0});
        } else {
            split_blocks.push_back(b);
            split_begin.push_back(nslots);
            for (int64_t k = 0; k < c; k += K) {
                items.push_back({bxi, byi, (int32_t)k, (int32_t)std::min<int64_t>(c, k + K), nslots, 0});
                nslots++;
            }
        }
    }
    split_begin.push_back(nslots);
    // heaviest items first (they are the tail otherwise)
    std::stable_sort(items.begin(), items.end(),
                     [](const Item& a, const Item& b) { return (a.k1 - a.k0) > (b.k1 - b.k0); });

    const size_t b_items = sizeof(Item) * items.size();
    const size_t b_scr = sizeof(double) * (size_t)kBlk * kBlk * (size_t)std::max(nslots, 1);
    const size_t b_sb = sizeof(int32_t) * (split_blocks.size() + 1);
    const size_t b_sbeg = sizeof(int32_t) * split_begin.size();
    Item* d_items = nullptr;
    int32_t *d_sb = nullptr, *d_sbeg = nullptr;
    if ((st = mgk_alloc(ctx, (void**)&d_items, b_items))) return st;
    if (nslots && (st = mgk_alloc(ctx, (void**)&P.scratch, b_scr))) { mgk_free(ctx, d_items, b_items); return st; }
    if (nslots && (st = mgk_alloc(ctx, (void**)&d_sb, b_sb))) {
        mgk_free(ctx, d_items, b_items); mgk_free(ctx, P.scratch, b_scr); return st;
    }
    if (nslots && (st = mgk_alloc(ctx, (void**)&d_sbeg, b_sbeg))) {
        mgk_free(ctx, d_items, b_items); mgk_free(ctx, P.scratch, b_scr); mgk_free(ctx, d_sb, b_sb); return st;
    }
    int rc = MGK_OK;
    do {
        if ((ce = cudaMemcpyAsync(d_items, items.data(), b_items, cudaMemcpyHostToDevice, s)) != cudaSuccess) break;
        if (nslots) {
            if ((ce = cudaMemcpyAsync(d_sb, split_blocks.data(), sizeof(int32_t) * split_blocks.size(),
                                      cudaMemcpyHostToDevice, s)) != cudaSuccess) break;
            if ((ce = cudaMemcpyAsync(d_sbeg, split_begin.data(), b_sbeg, cudaMemcpyHostToDevice, s)) != cudaSuccess) break;
        }
        P.items = d_items;
        const unsigned grid = (unsigned)items.size();
        cudaEventRecord(ctx->ev_a, s);
        if (fp64) {
            if (idx->varh) k_density_fp64<true><<<grid, kThreads, 0, s>>>(P);
            else k_density_fp64<false><<<grid, kThreads, 0, s>>>(P);
        } else if (d_evals) {
            if (idx->varh) k_density<true, true><<<grid, kThreads, 0, s>>>(P);
            else k_density<false, true><<<grid, kThreads, 0, s>>>(P);
        } else {
            if (idx->varh) k_density<true, false><<<grid, kThreads, 0, s>>>(P);
            else k_density<false, false><<<grid, kThreads, 0, s>>>(P);
        }
        cudaEventRecord(ctx->ev_b, s);
        if ((ce = cudaGetLastError()) != cudaSuccess) break;
        MGK_COUNT_LAUNCH(ctx, 2);  // plan + density
        if (nslots) {
            k_merge<<<(unsigned)split_blocks.size(), 256, 0, s>>>(P, d_sb, d_sbeg, nbx_t);
            if ((ce = cudaGetLastError()) != cudaSuccess) break;
            MGK_COUNT_LAUNCH(ctx, 1);
        }
        // the work list and scratch are freed below: wait for the kernels
        ce = cudaStreamSynchronize(s);
        if (ce == cudaSuccess) cudaEventElapsedTime(&ctx->last_density_ms, ctx->ev_a, ctx->ev_b);
    } while (0);
    if (ce != cudaSuccess) rc = mgk_cuda_fail(ctx, ce, "density");
    mgk_free(ctx, d_items, b_items);
    if (nslots) {
        mgk_free(ctx, P.scratch, b_scr);
        mgk_free(ctx, d_sb, b_sb);
        mgk_free(ctx, d_sbeg, b_sbeg);
    }
    return rc;
}
