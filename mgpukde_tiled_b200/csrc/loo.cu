// Leave-one-out log likelihood for a list of bandwidths in one launch.
//
// LogLikelihood (kde_cuda_kdtr_tiled.cu:3214-3299) recomputes the edge
// weights at h, scatters K_h(d) w_i e_i into every neighbour of i found by a
// k-d tree range search (DensityAtPointsKdtr, kde_kernel_kdtr.cu:681-804),
// subtracts the self term and takes logf(max(den, EPSILONDENSITY))
// (dCopyDensityValues, :806-830), then sums in float (ReductionSum,
// :1045-1111); MLE_FixedBandWidth (:3044-3093) calls it twice per
// golden-section step.  Here the density at query point j is gathered over
// its neighbours i != j:
//   loo_j(h) = sum_{i != j, d^2 < 9h^2} exp(-d^2 / 2h^2) / (h^2 TWO_PI) w_i e_i(h)
//   logL(h)  = sum_j log(max(loo_j(h), EPSILONDENSITY))
// for every h of a list, as one persistent launch over work items
// (h, group of 128 queries), heaviest h first, fed from a global item
// counter.  The points are indexed once per bandwidth octave (row-major bins
// of side in (0.375 h, 0.75 h] for the h that use the level), so the
// candidates of a group are one contiguous range per bin row; they arrive in
// batches of up to 128 (one bin row's range at a time) through a
// double-buffered TMA bulk copy into shared memory, and every thread (one
// query) scans them.  The cutoff is decided in FP32
// with a band around 9h^2 re-decided by the oracle's exact FP64 test, so the
// summed pair set is exactly the oracle's; terms are FP32 (an exp2 by range
// reduction and a polynomial, free of the systematic bias an approximate
// special-function exp2 would add to every one of the sum's terms), summed
// per batch and added into a Kahan-compensated FP32 accumulator; the per-query log is FP64, and the per-group and per-h sums
// are fixed-order FP64 trees (bitwise reproducible).  The argmax is taken on
// the device.  The whole sequence (edge weights for every h, the gather, the
// sums, the argmax) is captured once into a CUDA graph and replayed, with the
// bandwidths read from device memory, so a golden-section step is one graph
// launch.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "mgk_internal.cuh"

namespace {

constexpr int kLooQ = 128;    // queries (threads) per work item
// candidates per staged batch (at most one per thread, which reads its
// candidate's weight): with the scan unrolled by 8, 32, 64 and 128 gave
// 271, 257 and 251 ms for the 64-bandwidth selection (C2)
constexpr int kLooB = 128;
static_assert(kLooB <= kLooQ, "one thread per staged candidate");
constexpr int kMaxLev = 16;   // bandwidth octaves
constexpr long long kLooSpin = 1ll << 24;

struct LevelDesc {
    const MgkPt* pts;
    const int32_t* bin_start;
    const int32_t* perm;
    const int32_t* qord;  // query order: record positions in Z-order of the bins
    double ox, oy, side, inv_side;
    int64_t nbx, nby;
    double quantum;       // coordinate quantum of the records' hi/lo split
};

// Rejects most out-of-cutoff candidates on their hi parts (4 instructions)
// before the exact pair arithmetic.
#ifndef MGK_LOO_PREFILTER
#define MGK_LOO_PREFILTER 1
#endif
// candidates per trip of the scan loop: 8 measured fastest on the
// 64-bandwidth selection (C2: 317, 290, 282, 271, 274 and 290 ms at 1, 2, 4,
// 8, 16 and 32; the compiler's own choice gave 290)
#ifndef MGK_LOO_UNROLL
#define MGK_LOO_UNROLL 8
#endif
constexpr int kLooUnroll = MGK_LOO_UNROLL;

struct LooParams {
    const LevelDesc* lev;  // [nlev], device
    double side[kMaxLev];  // bin side of each level
    int nlev;
    int64_t n;
    int ngroups;
    int g0, gcount;       // this share's query groups [g0, g0 + gcount) (all groups: 0, ngroups)
    int nh;
    const float* hgrid;   // [nh]
    int* korder;          // [nh] processing order (largest h first)
    int* klevel;          // [nh] level of each h
    // edge weights, or null (no edge correction): e_i(h_k) of point i (input
    // order) is ew[(i / ew_chunk) * ew_cstride + k * ew_chunk + i % ew_chunk],
    // i.e. chunks of ew_chunk points, each nh rows of ew_chunk floats (one
    // chunk of n points, [nh][n], in a single-process batch)
    const float* ew;
    int64_t ew_chunk, ew_cstride;
    double* part;         // [nh][gcount]
    unsigned* counter;    // work-item queue head
    unsigned long long* evals;
    unsigned long long* err;
};

// ---- TMA bulk copy + mbarrier (sm_90+ PTX) ---------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
    for (long long i = 0; i < kLooSpin; i++)
        if (mbar_try_wait(b, parity)) return true;
    return false;
}

__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); i++) t += sh[i];
    return t;
}

// Level and processing order of every h (one CTA; nh is small).
__global__ void k_loo_prep(LooParams P) {
    for (int k = threadIdx.x; k < P.nh; k += blockDim.x) {
        const float h = P.hgrid[k];
        int L = 0;
        for (int l = 1; l < P.nlev; l++)
            if (P.side[l] <= 0.75 * (double)h) L = l;
        int rank = 0;
        for (int j = 0; j < P.nh; j++) {
            const float hj = P.hgrid[j];
            rank += (hj > h) || (hj == h && j < k);
        }
        P.klevel[k] = L;
        P.korder[rank] = k;
    }
}

__global__ void __launch_bounds__(kLooQ) k_loo_multi(LooParams P) {
    __shared__ __align__(128) MgkPt stage[2][kLooB];
    __shared__ float sw[2][kLooB];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ double red[kLooQ / 32];
    __shared__ float bb[4][kLooQ / 32];
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        mbar_init(&mbar[0], 1);
        mbar_init(&mbar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned ph0 = 0u, ph1 = 0u;  // mbarrier phase parities of the two buffers
    const unsigned total = (unsigned)P.nh * (unsigned)P.gcount;
    unsigned long long cnt_all = 0;
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(P.counter, 1u);
        __syncthreads();
        const unsigned item = (unsigned)s_item;
        if (item >= total) break;
        const int k = P.korder[item / (unsigned)P.gcount];
        const int grp = P.g0 + (int)(item % (unsigned)P.gcount);
        const LevelDesc L = P.lev[P.klevel[k]];
        const float h = P.hgrid[k];
        const double h2 = mgk_h2(h);
        const double cut = MGK_CUT * h2;
        const float cutf = (float)cut;
        const float epsd2 = cutf * 4e-6f;
        // log2(e) / (2 h^2) as a float pair: a one-float scale would bias every
        // exponent of the batch the same way
        const double k2 = MGK_LOG2E / (2.0 * h2);
        const float k2h = (float)k2, k2l = (float)(k2 - (double)k2h);
        const double reach = sqrt(cut) * (1.0 + 1e-9);
        // squared hi-part distance beyond which a candidate is surely outside
        // the cutoff (|lo parts| <= q / 2 each; 1e-5 covers the float rounding)
        const float far2 = (float)((reach + 2.0 * L.quantum) * (reach + 2.0 * L.quantum) * (1.0 + 1e-5));
        const float* ewk = P.ew ? P.ew + (int64_t)k * P.ew_chunk : nullptr;

        // this item's query
        // the group's queries: 128 consecutive records of the Z-order, a
        // compact patch of bins (row-major runs would be long thin strips)
        const int64_t qk = (int64_t)grp * kLooQ + tid;
        const bool qv = qk < P.n;
        const int64_t qpos = qv ? (int64_t)L.qord[qk] : -1;
        MgkPt q{};
        if (qv) q = L.pts[qpos];
        const float qx = q.xh + q.xl, qy = q.yh + q.yl;
        // bounding box of the group's queries
        float mnx = qv ? qx : FLT_MAX, mxx = qv ? qx : -FLT_MAX, mny = qv ? qy : FLT_MAX, mxy = qv ? qy : -FLT_MAX;
        for (int o = 16; o; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        if (lane == 0) {
            bb[0][warp] = mnx;
            bb[1][warp] = mxx;
            bb[2][warp] = mny;
            bb[3][warp] = mxy;
        }
        __syncthreads();
        for (int i = 0; i < kLooQ / 32; i++) {
            mnx = fminf(mnx, bb[0][i]);
            mxx = fmaxf(mxx, bb[1][i]);
            mny = fminf(mny, bb[2][i]);
            mxy = fmaxf(mxy, bb[3][i]);
        }
        const int64_t bx0 = mgk_max64(0, (int64_t)floor(((double)mnx - reach - L.ox) * L.inv_side));
        const int64_t bx1 = mgk_min64(L.nbx - 1, (int64_t)floor(((double)mxx + reach - L.ox) * L.inv_side));
        const int64_t by0 = mgk_max64(0, (int64_t)floor(((double)mny - reach - L.oy) * L.inv_side));
        const int64_t by1 = mgk_min64(L.nby - 1, (int64_t)floor(((double)mxy + reach - L.oy) * L.inv_side));

        float s = 0.0f, c = 0.0f;
        unsigned cnt = 0;
        // candidate stream: batches of <= kLooB within one bin row
        int64_t by = by0, pos = 0, end = 0;
        auto next = [&](int64_t& src) -> int {
            while (pos >= end) {
                if (by > by1 || bx0 > bx1) return 0;
                pos = L.bin_start[by * L.nbx + bx0];
                end = L.bin_start[by * L.nbx + bx1 + 1];
                by++;
            }
            const int m = (int)mgk_min64(kLooB, end - pos);
            src = pos;
            pos += m;
            return m;
        };
        int64_t src = 0, nsrc = 0;
        int m = next(src);
        int buf = 0;
        if (m > 0 && tid == 0) {
            mbar_arrive_tx(&mbar[0], (unsigned)(m * sizeof(MgkPt)));
            bulk_g2s(&stage[0][0], L.pts + src, (unsigned)(m * sizeof(MgkPt)), &mbar[0]);
        }
        while (m > 0) {
            const int nm = next(nsrc);
            if (nm > 0 && tid == 0) {
                mbar_arrive_tx(&mbar[buf ^ 1], (unsigned)(nm * sizeof(MgkPt)));
                bulk_g2s(&stage[buf ^ 1][0], L.pts + nsrc, (unsigned)(nm * sizeof(MgkPt)), &mbar[buf ^ 1]);
            }
            if (tid < m) {
                const int64_t i = src + tid;
                float e = 1.0f;
                if (ewk) {
                    const int64_t pi = L.perm[i], ch = pi / P.ew_chunk;
                    e = ewk[ch * P.ew_cstride + (pi - ch * P.ew_chunk)];
                }
                sw[buf][tid] = L.pts[i].wk * e;
            }
            const unsigned par = buf ? ph1 : ph0;
            const bool ok = mbar_wait(&mbar[buf], par);
            if (__syncthreads_or(!ok)) {
                // a staging wait ran out: flag it and give the copies in
                // flight a second bounded wait before the CTA goes away
                if (tid == 0) {
                    atomicExch(P.err, 1ull);
                    mbar_wait(&mbar[buf], par);
                    if (nm > 0) mbar_wait(&mbar[buf ^ 1], buf ? ph0 : ph1);
                }
                __syncthreads();
                return;
            }
            if (buf) ph1 ^= 1u;
            else ph0 ^= 1u;
            if (qv) {
                float part = 0.0f;
                const MgkPt* st = stage[buf];
#pragma unroll kLooUnroll
                for (int t = 0; t < m; t++) {
                    const float4 cp = *reinterpret_cast<const float4*>(&st[t]);
#if MGK_LOO_PREFILTER
                    // the hi parts alone first: their difference is exact and
                    // the lo parts move d by at most 2 quanta, so a candidate
                    // beyond far2 is outside the cutoff (2 of 3 tested are)
                    const float dxh = __fsub_rn(cp.x, q.xh), dyh = __fsub_rn(cp.y, q.yh);
                    if (__fmaf_rn(dxh, dxh, __fmul_rn(dyh, dyh)) > far2) continue;
#endif
                    const float dx = __fadd_rn(__fsub_rn(cp.x, q.xh), __fsub_rn(cp.z, q.xl));
                    const float dy = __fadd_rn(__fsub_rn(cp.y, q.yh), __fsub_rn(cp.w, q.yl));
                    const float d2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                    bool in = d2 < cutf;
                    if (fabsf(d2 - cutf) <= epsd2)  // near the cutoff: the oracle's FP64 decision
                        in = mgk_d2_exact(qx, qy, cp.x + cp.z, cp.y + cp.w) < cut;
                    if (in && src + t != qpos) {
                        const float a = __fmaf_rn(d2, k2h, __fmul_rn(d2, k2l));
                        part = __fmaf_rn(mgk_exp2_neg_poly(a), sw[buf][t], part);
                        cnt++;
                    }
                }
                const float y = part - c;
                const float tt = s + y;
                c = (tt - s) - y;
                s = tt;
            }
            __syncthreads();  // stage[buf] and sw[buf] are reused two batches on
            m = nm;
            src = nsrc;
            buf ^= 1;
        }
        double lg = 0.0;
        if (qv) {
            const double loo = ((double)s - (double)c) / (h2 * (double)MGK_TWO_PI_F);
            const double fl = (double)MGK_EPS_DENSITY_F;
            lg = log(loo > fl ? loo : fl);
        }
        const double sum = block_sum_fixed(lg, red);
        if (tid == 0) P.part[(int64_t)k * P.gcount + (grp - P.g0)] = sum;
        cnt_all += cnt;
        __syncthreads();  // s_item is rewritten next
    }
    if (P.evals) {
        for (int o = 16; o; o >>= 1) cnt_all += __shfl_xor_sync(0xffffffffu, cnt_all, o);
        if (lane == 0 && cnt_all) atomicAdd(P.evals, cnt_all);
    }
}

// logL[k] = fixed-order sum of the group partials of h_k (one CTA per h).
__global__ void k_loo_finish(const double* __restrict__ part, int ngroups, double* __restrict__ logl) {
    __shared__ double sh[256];
    const int k = blockIdx.x;
    double v = 0.0;
    for (int i = threadIdx.x; i < ngroups; i += blockDim.x) v += part[(int64_t)k * ngroups + i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) logl[k] = sh[0];
}

// First index of the largest logL (ties resolve to the lower index).
__global__ void k_argmax(const double* __restrict__ logl, int nh, int* __restrict__ best) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int b = 0;
        for (int k = 1; k < nh; k++)
            if (logl[k] > logl[b]) b = k;
        *best = b;
    }
}

}  // namespace

// ---- the batch object ------------------------------------------------------
struct mgk_loo_batch {
    mgk_ctx* ctx = nullptr;
    const mgk_points* pts = nullptr;
    const mgk_raster* mask = nullptr;
    int64_t n = 0;
    int nh = 0;
    int ngroups = 0;
    int g0 = 0, gcount = 0;  // the share's query groups
    std::vector<mgk_index*> lev;
    std::vector<int32_t*> qord;  // per level
    float* d_h = nullptr;
    float* d_ew = nullptr;
    LevelDesc* d_lev = nullptr;
    cudaStream_t cap = nullptr;  // capture stream
    int* d_korder = nullptr;
    int* d_klevel = nullptr;
    double* d_part = nullptr;
    double* d_logl = nullptr;
    int* d_best = nullptr;
    unsigned* d_counter = nullptr;
    unsigned long long* d_evals = nullptr;  // [0] edge, [1] loo
    unsigned long long* d_err = nullptr;
    float* h_h = nullptr;       // pinned
    double* h_logl = nullptr;   // pinned: nh logL, then the argmax and the eval counts
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    LooParams P{};
    size_t bytes_ew = 0, bytes_part = 0;
};

static int loo_enqueue(mgk_loo_batch* B) {
    mgk_ctx* ctx = B->ctx;
    cudaStream_t s = ctx->stream;
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(B->d_counter, 0, sizeof(unsigned), s));
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(B->d_evals, 0, 2 * sizeof(unsigned long long), s));
    MGK_CHECK_CUDA(ctx, cudaMemsetAsync(B->d_err, 0, sizeof(unsigned long long), s));
    if (B->mask) {
        int st = mgk_launch_edge_weights_multi(ctx, B->n, B->pts->x, B->pts->y, nullptr, 0.0f, B->d_h, B->nh,
                                               B->pts->dist2, B->mask, B->d_ew, B->n, B->d_evals);
        if (st) return st;
    }
    k_loo_prep<<<1, 256, 0, s>>>(B->P);
    const int occ = 8;  // resident CTAs of 128 threads per SM targeted by the persistent grid
    const unsigned items = (unsigned)B->nh * (unsigned)std::max(B->P.gcount, 1);
    const unsigned grid = std::max(1u, std::min(items, (unsigned)(ctx->sm_count * occ)));
    k_loo_multi<<<grid, kLooQ, 0, s>>>(B->P);
    k_loo_finish<<<B->nh, 256, 0, s>>>(B->d_part, B->P.gcount, B->d_logl);
    k_argmax<<<1, 32, 0, s>>>(B->d_logl, B->nh, B->d_best);
    MGK_CHECK_LAUNCH(ctx, "loo batch");
    MGK_COUNT_LAUNCH(ctx, 4);
    return MGK_OK;
}

void mgk_loo_batch_destroy(mgk_loo_batch* B) {
    if (!B) return;
    mgk_ctx* c = B->ctx;
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    if (B->cap) cudaStreamDestroy(B->cap);
    mgk_free(c, B->d_lev, sizeof(LevelDesc) * kMaxLev);
    for (int32_t* q : B->qord) mgk_free(c, q, sizeof(int32_t) * (size_t)std::max<int64_t>(B->n, 1));
    for (mgk_index* i : B->lev) mgk_index_destroy(i);
    const size_t nh = (size_t)B->nh;
    mgk_free(c, B->d_h, sizeof(float) * nh);
    mgk_free(c, B->d_ew, B->bytes_ew);
    mgk_free(c, B->d_korder, sizeof(int) * nh);
    mgk_free(c, B->d_klevel, sizeof(int) * nh);
    mgk_free(c, B->d_part, B->bytes_part);
    mgk_free(c, B->d_logl, sizeof(double) * nh);
    mgk_free(c, B->d_best, sizeof(int));
    mgk_free(c, B->d_counter, sizeof(unsigned));
    mgk_free(c, B->d_evals, 2 * sizeof(unsigned long long));
    mgk_free(c, B->d_err, sizeof(unsigned long long));
    if (B->h_h) cudaFreeHost(B->h_h);
    if (B->h_logl) cudaFreeHost(B->h_logl);
    delete B;
}

// Plans a batch of nh bandwidths within [h_lo, h_hi]: one point index per
// bandwidth octave, buffers, and the captured graph.
int mgk_loo_batch_create(mgk_ctx* c, const mgk_points* p, const mgk_raster* r, float h_lo, float h_hi, int nh,
                         mgk_loo_batch** out) {
    return mgk_loo_batch_create_share(c, p, r, h_lo, h_hi, nh, 0, 1, nullptr, 0, out, true);
}

// Share `part` of `nparts` of a batch: the query groups
// [part G / nparts, (part + 1) G / nparts) of every h, G = ceil(n / 128).
// ew_ext (device, optional, with r == NULL): the edge weights of every point
// and h in chunks of ew_chunk points, each nh rows of ew_chunk floats.
int mgk_loo_batch_create_share(mgk_ctx* c, const mgk_points* p, const mgk_raster* r, float h_lo, float h_hi,
                               int nh, int part, int nparts, const float* ew_ext, int64_t ew_chunk,
                               mgk_loo_batch** out, bool replay) {
    mgk_loo_batch* B = new (std::nothrow) mgk_loo_batch();
    if (!B) return mgk_fail(c, MGK_ERR_INVALID, "loo batch: out of host memory");
    B->ctx = c;
    B->pts = p;
    B->mask = r;
    B->n = p->n;
    B->nh = nh;
    B->ngroups = (int)((p->n + kLooQ - 1) / kLooQ);
    B->g0 = (int)((int64_t)B->ngroups * part / nparts);
    B->gcount = (int)((int64_t)B->ngroups * (part + 1) / nparts) - B->g0;
    int st = MGK_OK;
    // levels: bin sides 0.75 h_lo * 2^l up to the side for h_hi
    mgk_points view = *p;  // index over w only; e(h) is applied per h
    view.has_ew = false;
    view.h = nullptr;
    const int nlev = std::min(kMaxLev, 1 + std::max(0, (int)std::ceil(std::log2((double)h_hi / (double)h_lo))));
    for (int l = 0; l < nlev && st == MGK_OK; l++) {
        const float side = (float)(0.75 * (double)h_lo * std::ldexp(1.0, l));
        mgk_index* idx = nullptr;
        st = mgk_index_build(c, &view, h_lo, side, &idx);
        if (st == MGK_OK) {
            B->lev.push_back(idx);
            int32_t* q = nullptr;
            st = mgk_alloc(c, (void**)&q, sizeof(int32_t) * (size_t)std::max<int64_t>(p->n, 1));
            if (st == MGK_OK) {
                B->qord.push_back(q);
                st = mgk_index_zorder(c, idx, q);
            }
            if (st) break;
            // levels whose side was raised to the bin-count limit repeat the previous one
            if (l > 0 && idx->side <= B->lev[l - 1]->side) break;
        }
    }
    const size_t n1 = (size_t)std::max<int64_t>(p->n, 1);
    B->bytes_ew = r ? sizeof(float) * n1 * (size_t)nh : 16;
    B->bytes_part = sizeof(double) * (size_t)nh * (size_t)std::max(B->gcount, 1);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_h, sizeof(float) * nh);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_ew, B->bytes_ew);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_korder, sizeof(int) * nh);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_klevel, sizeof(int) * nh);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_part, B->bytes_part);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_logl, sizeof(double) * nh);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_best, sizeof(int));
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_counter, sizeof(unsigned));
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_evals, 2 * sizeof(unsigned long long));
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_err, sizeof(unsigned long long));
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&B->d_lev, sizeof(LevelDesc) * kMaxLev);
    if (st == MGK_OK && r) st = mgk_raster_runs(c, const_cast<mgk_raster*>(r));
    if (st == MGK_OK && cudaMallocHost((void**)&B->h_h, sizeof(float) * nh) != cudaSuccess)
        st = mgk_fail(c, MGK_ERR_CUDA, "loo batch: pinned allocation");
    if (st == MGK_OK && cudaMallocHost((void**)&B->h_logl, sizeof(double) * (nh + 3)) != cudaSuccess)
        st = mgk_fail(c, MGK_ERR_CUDA, "loo batch: pinned allocation");
    if (st) {
        mgk_loo_batch_destroy(B);
        return st;
    }
    LooParams& P = B->P;
    P.nlev = (int)B->lev.size();
    LevelDesc hl[kMaxLev];
    for (int l = 0; l < P.nlev; l++) {
        const mgk_index* I = B->lev[l];
        hl[l] = LevelDesc{I->pts, I->bin_start, I->perm, B->qord[l], I->ox, I->oy, I->side, 1.0 / I->side, I->nbx,
                          I->nby, std::ldexp(1.0, -I->qexp)};
        P.side[l] = I->side;
    }
    if (cudaMemcpy(B->d_lev, hl, sizeof(LevelDesc) * P.nlev, cudaMemcpyHostToDevice) != cudaSuccess) {
        mgk_loo_batch_destroy(B);
        return mgk_fail(c, MGK_ERR_CUDA, "loo batch: level table");
    }
    P.lev = B->d_lev;
    P.n = p->n;
    P.ngroups = B->ngroups;
    P.g0 = B->g0;
    P.gcount = B->gcount;
    P.nh = nh;
    P.hgrid = B->d_h;
    P.korder = B->d_korder;
    P.klevel = B->d_klevel;
    if (r) {
        P.ew = B->d_ew;
        P.ew_chunk = std::max<int64_t>(p->n, 1);
    } else if (ew_ext) {
        P.ew = ew_ext;
        P.ew_chunk = std::max<int64_t>(ew_chunk, 1);
    } else {
        P.ew = nullptr;
        P.ew_chunk = 1;
    }
    P.ew_cstride = P.ew_chunk * (int64_t)nh;
    P.part = B->d_part;
    P.counter = B->d_counter;
    P.evals = B->d_evals + 1;
    P.err = B->d_err;
    // capture the sequence into a graph on a private stream (the graph is
    // then launched into the context's stream); if capture fails, or the
    // batch runs once (replay false: capture and instantiation would cost
    // more than they save), the batch launches its kernels directly
    if (replay && cudaStreamSynchronize(c->stream) == cudaSuccess &&
        cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking) == cudaSuccess &&
        cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        cudaStream_t keep = c->stream;
        const uint64_t l0 = c->launches;
        c->stream = B->cap;
        const int est = loo_enqueue(B);
        c->stream = keep;
        c->launches = l0;  // counted at each replay
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(B->cap, &g);
        if (est == MGK_OK && ce == cudaSuccess && g) {
            B->graph = g;
            if (cudaGraphInstantiate(&B->exec, g, 0) != cudaSuccess) B->exec = nullptr;
        } else if (g) {
            cudaGraphDestroy(g);
        }
        cudaGetLastError();
    }
    *out = B;
    return MGK_OK;
}

// Scores the nh bandwidths hs (host) of a planned batch: logL, argmax and the
// edge and LOO eval counts.
int mgk_loo_batch_run(mgk_loo_batch* B, const float* hs, double* logl, int* best, int64_t* edge_evals,
                      int64_t* loo_evals) {
    mgk_ctx* c = B->ctx;
    cudaStream_t s = c->stream;
    for (int k = 0; k < B->nh; k++) B->h_h[k] = hs[k];
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(B->d_h, B->h_h, sizeof(float) * B->nh, cudaMemcpyHostToDevice, s));
    MGK_CHECK_CUDA(c, cudaEventRecord(c->ev_a, s));
    if (B->exec) {
        MGK_CHECK_CUDA(c, cudaGraphLaunch(B->exec, s));
        MGK_COUNT_LAUNCH(c, 4 + (B->mask ? 1 : 0));
    } else {
        int st = loo_enqueue(B);
        if (st) return st;
    }
    MGK_CHECK_CUDA(c, cudaEventRecord(c->ev_b, s));
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(B->h_logl, B->d_logl, sizeof(double) * B->nh, cudaMemcpyDeviceToHost, s));
    unsigned long long* tail = reinterpret_cast<unsigned long long*>(B->h_logl + B->nh);
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(tail, B->d_evals, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(tail + 2, B->d_err, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    int* hb = reinterpret_cast<int*>(c->h_counter);
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(hb, B->d_best, sizeof(int), cudaMemcpyDeviceToHost, s));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(s));
    if (tail[2]) return mgk_fail(c, MGK_ERR_TIMEOUT, "loo batch: a staging wait timed out");
    for (int k = 0; k < B->nh; k++) logl[k] = B->h_logl[k];
    if (best) *best = *hb;
    if (edge_evals) *edge_evals = (int64_t)tail[0];
    if (loo_evals) *loo_evals = (int64_t)tail[1];
    c->last_loo_evals[0] = (int64_t)tail[0];
    c->last_loo_evals[1] = (int64_t)tail[1];
    cudaEventElapsedTime(&c->last_loo_ms, c->ev_a, c->ev_b);
    return MGK_OK;
}
