// Adaptive bandwidths (h_option 2): Hooke-Jeeves search over (h0, alpha).
//
// The reference (main, kde_cuda_kdtr_tiled.cu:548-573) starts from the
// rule-of-thumb h0 with alpha0 = -0.5 and searches (hooke_jeeves /
// hj_likelihood, :3677-3785) for the (h, alpha) maximising
// LogLikelihood(h, alpha) (CPU branch :3553-3650):
//   1. edge weights e(h) at the fixed h,
//   2. pilot density at every point, itself included:
//        den0_j = sum_{i, d^2 < 9h^2} K_h(d) w_i e_i(h),
//   3. hs_i = h (den0_i / gml)^alpha, gml the geometric mean of den0 (compGML),
//   4. edge weights e(hs) at the per-point bandwidths,
//   5. leave-one-out density with the bandwidth of each source point:
//        den1_j = sum_{i != j, d^2 < 9 hs_i^2} K_{hs_i}(d) w_i e_i(hs),
//   6. logL = sum_j log max(den1_j, EPSILONDENSITY).
// After the search the bandwidths of the optimum are computed once more
// (steps 1-3) and used for the density raster.
//
// On the device: steps 1 and 4 are k_edge_rows; steps 2 and 5 are
// k_point_density over a cell-binned index of the points (fixed-h index for
// the pilot, per-point-h index for the LOO sum), one thread per query, the
// candidates staged through shared memory, the cutoff decided in FP32 with a
// band re-decided by the oracle's FP64 test, terms from the unbiased
// polynomial exp2, Kahan-compensated FP32 partials and an FP64 result per
// point; the geometric mean, the bandwidths and the log sum are FP64 on the
// device (fixed-order reductions).  The search itself runs on the host with
// the reference's float step arithmetic and its bookkeeping of the five
// likelihoods.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>

#include "mgk_internal.cuh"

namespace {

constexpr int kPdQ = 128;  // queries (threads) per CTA
constexpr int kPdB = 32;   // candidates per staged batch

// psum[y][q] = sum over candidates i (the points of the index within reach
// of the CTA's 128 consecutive queries, in the bin rows y, y + nsplit, ... of
// the window, y = blockIdx.y) of [in cutoff] K w_i e_i, unnormalised; the
// query itself is included when SELF.  Fixed h: terms exp2(-d^2 k2) w e;
// per-point h (VARH): the candidate's own k2 and cutoff, weights already
// carry 1/(h_i^2 TWO_PI).  Splitting the rows over nsplit CTAs gives a
// launch enough CTAs for the whole GPU when there are few queries.
//
// Per-point h: the window is the group's bounding box grown by the largest
// reach of all points, but in each bin row only the span from the first to
// the last bin whose own largest reach (bin_r2: 9 h^2 of its widest point)
// can touch the box is read, so points with small h far from the group are
// never tested.
// candidates per trip of the scan loop (8: 49.5 ms per adaptive search
// against 50.6 ms at the compiler's own choice, 49.7 at 4 and 16)
#ifndef MGK_PD_UNROLL
#define MGK_PD_UNROLL 8
#endif
constexpr int kPdUnroll = MGK_PD_UNROLL;

template <bool VARH, bool SELF>
__global__ void __launch_bounds__(kPdQ) k_point_density(int64_t n, const MgkPt* __restrict__ pts,
                                                        const int32_t* __restrict__ bin_start, double ox,
                                                        double oy, double side, int64_t nbx, int64_t nby,
                                                        double reach, double h2, const float* __restrict__ bin_r2,
                                                        double quantum, double* __restrict__ psum,
                                                        unsigned long long* __restrict__ evals) {
    __shared__ __align__(16) MgkPt st[kPdB];
    __shared__ float bb[4][kPdQ / 32];
    __shared__ int s_span[2];
    const double inv_side = 1.0 / side;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t qpos = (int64_t)blockIdx.x * kPdQ + tid;
    const bool qv = qpos < n;
    MgkPt q{};
    if (qv) q = pts[qpos];
    const float qx = q.xh + q.xl, qy = q.yh + q.yl;
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
    for (int i = 0; i < kPdQ / 32; i++) {
        mnx = fminf(mnx, bb[0][i]);
        mxx = fmaxf(mxx, bb[1][i]);
        mny = fminf(mny, bb[2][i]);
        mxy = fmaxf(mxy, bb[3][i]);
    }
    const int64_t bx0 = mgk_max64(0, (int64_t)floor(((double)mnx - reach - ox) * inv_side));
    const int64_t bx1 = mgk_min64(nbx - 1, (int64_t)floor(((double)mxx + reach - ox) * inv_side));
    const int64_t by0 = mgk_max64(0, (int64_t)floor(((double)mny - reach - oy) * inv_side));
    const int64_t by1 = mgk_min64(nby - 1, (int64_t)floor(((double)mxy + reach - oy) * inv_side));
    // fixed-h constants
    const double cut = MGK_CUT * h2;
    const float cutf = (float)cut;
    const double k2 = MGK_LOG2E / (2.0 * h2);
    const float k2h = (float)k2, k2l = (float)(k2 - (double)k2h);
    // squared hi-part distance beyond which a candidate is outside its cutoff:
    // the hi parts' difference is exact and the lo parts move d by at most
    // two quanta, so (3h + 2q)^2 = 9h^2 + 12 h q + 4 q^2 bounds it (h <= the
    // widest reach / 3; 1e-5 covers the float rounding).  Fixed h: one bound.
    const float far2 = (float)((reach + 2.0 * quantum) * (reach + 2.0 * quantum) * (1.0 + 1e-5));
    const float far_add = (float)((4.0 * reach * quantum + 4.0 * quantum * quantum) * (1.0 + 1e-5));
    float s = 0.0f, c = 0.0f;
    unsigned cnt = 0;
    for (int64_t by = by0 + blockIdx.y; by <= by1 && bx0 <= bx1; by += gridDim.y) {
        int64_t lo = bx0, hi = bx1;
        if (VARH) {
            __syncthreads();  // s_span of the previous row has been read
            if (tid == 0) {
                s_span[0] = INT_MAX;
                s_span[1] = -1;
            }
            __syncthreads();
            const double ry0 = oy + (double)by * side, ry1 = ry0 + side;
            const double ddy = fmax(0.0, fmax(ry0 - (double)mxy, (double)mny - ry1));
            for (int64_t bx = bx0 + tid; bx <= bx1; bx += kPdQ) {
                const float r2 = bin_r2[by * nbx + bx];
                if (r2 < 0.0f) continue;  // empty bin
                const double rx0 = ox + (double)bx * side, rx1 = rx0 + side;
                const double ddx = fmax(0.0, fmax(rx0 - (double)mxx, (double)mnx - rx1));
                // a margin over the bin edges' rounding and the float h^2
                if (ddx * ddx + ddy * ddy <= (double)r2 * (1.0 + 1e-5) + 1e-6 * side * side) {
                    atomicMin(&s_span[0], (int)(bx - bx0));
                    atomicMax(&s_span[1], (int)(bx - bx0));
                }
            }
            __syncthreads();
            if (s_span[1] < 0) continue;  // no bin of the row reaches the group (uniform)
            lo = bx0 + s_span[0];
            hi = bx0 + s_span[1];
        }
        const int64_t sb = bin_start[by * nbx + lo], se = bin_start[by * nbx + hi + 1];
        for (int64_t base = sb; base < se; base += kPdB) {
            const int m = (int)mgk_min64(kPdB, se - base);
            __syncthreads();
            if (tid < m) st[tid] = pts[base + tid];
            __syncthreads();
            if (!qv) continue;
            float part = 0.0f;
#pragma unroll kPdUnroll
            for (int t = 0; t < m; t++) {
                const MgkPt p = st[t];
                const float dxh = __fsub_rn(p.xh, q.xh), dyh = __fsub_rn(p.yh, q.yh);
                const float lim = VARH ? __fmaf_rn(9.0f * p.hh, 1.00001f, far_add) : far2;
                if (__fmaf_rn(dxh, dxh, __fmul_rn(dyh, dyh)) > lim) continue;
                const float dx = __fadd_rn(__fsub_rn(p.xh, q.xh), __fsub_rn(p.xl, q.xl));
                const float dy = __fadd_rn(__fsub_rn(p.yh, q.yh), __fsub_rn(p.yl, q.yl));
                const float d2 = __fmaf_rn(dx, dx, __fmul_rn(dy, dy));
                const float cf = VARH ? 9.0f * p.hh : cutf;
                bool in = d2 < cf;
                if (fabsf(d2 - cf) <= cf * 4e-6f)  // near the cutoff: the oracle's FP64 decision
                    in = mgk_d2_exact(qx, qy, p.xh + p.xl, p.yh + p.yl) < (VARH ? MGK_CUT * (double)p.hh : cut);
                if (!SELF && base + t == qpos) in = false;
                if (in) {
                    const float a = VARH ? __fmaf_rn(d2, p.k2h, __fmul_rn(d2, p.k2l))
                                         : __fmaf_rn(d2, k2h, __fmul_rn(d2, k2l));
                    part = __fmaf_rn(mgk_exp2_neg_poly(a), p.wk, part);
                    cnt++;
                }
            }
            const float y = part - c;
            const float tt = s + y;
            c = (tt - s) - y;
            s = tt;
        }
    }
    if (qv) psum[(int64_t)blockIdx.y * n + qpos] = (double)s - (double)c;
    if (evals) {
        for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0 && cnt) atomicAdd(evals, (unsigned long long)cnt);
    }
}

// den[perm[q]] = the nsplit partials of query q summed in order (times
// 1/(h^2 TWO_PI) for a fixed h), and part[CTA] = the CTA's fixed-order sum of
// log(max(den, floor_v)).
__global__ void __launch_bounds__(kPdQ) k_pd_combine(int64_t n, int nsplit, const double* __restrict__ psum,
                                                     const int32_t* __restrict__ perm, bool varh, double h2,
                                                     double floor_v, double* __restrict__ den,
                                                     double* __restrict__ part) {
    __shared__ double s_lg[kPdQ / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t q = (int64_t)blockIdx.x * kPdQ + tid;
    double lg = 0.0;
    if (q < n) {
        double v = 0.0;
        for (int y = 0; y < nsplit; y++) v += psum[(int64_t)y * n + q];
        if (!varh) v /= h2 * (double)MGK_TWO_PI_F;
        den[perm[q]] = v;
        lg = log(v > floor_v ? v : floor_v);
    }
    for (int o = 16; o; o >>= 1) lg += __shfl_xor_sync(0xffffffffu, lg, o);
    if (lane == 0) s_lg[warp] = lg;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int i = 0; i < kPdQ / 32; i++) t += s_lg[i];
        part[blockIdx.x] = t;
    }
}

// out[0] = sum of the per-CTA partials in a fixed order (one CTA).
__global__ void k_sum_parts(int64_t g, const double* __restrict__ part, double* __restrict__ out) {
    __shared__ double sh[256];
    double a = 0.0;
    for (int64_t i = threadIdx.x; i < g; i += blockDim.x) a += part[i];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = sh[0];
}

// hs_i = h (den0_i / gml)^alpha with gml = exp(logsum / n).
__global__ void k_adaptive_h(int64_t n, const double* __restrict__ den0, const double* __restrict__ logsum, float h,
                             float alpha, float* __restrict__ hs) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double gml = exp(logsum[0] / (double)n);
    hs[i] = (float)((double)h * pow(den0[i] / gml, (double)alpha));
}

// Per bin: 9 h^2 of its widest point (-1 for an empty bin).
__global__ void k_bin_reach2(int64_t nbins, const int32_t* __restrict__ bin_start, const MgkPt* __restrict__ pts,
                             float* __restrict__ r2) {
    const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (b >= nbins) return;
    float m = -1.0f;
    for (int64_t t = bin_start[b]; t < bin_start[b + 1]; t++) m = fmaxf(m, pts[t].hh);
    r2[b] = m < 0.0f ? -1.0f : 9.0f * m;
}

// Counters of a likelihood computation: context counter slots 5 (edge-mask
// cells) and 6 (point pairs inside the cutoff), accumulated over all steps.
unsigned long long* edge_count(mgk_ctx* c) { return c->d_counter + 5; }
unsigned long long* pair_count(mgk_ctx* c) { return c->d_counter + 6; }

int count_begin(mgk_ctx* c) {
    MGK_CHECK_CUDA(c, cudaMemsetAsync(c->d_counter + 5, 0, 2 * sizeof(unsigned long long), c->stream));
    MGK_CHECK_CUDA(c, cudaEventRecord(c->ev_a, c->stream));
    return MGK_OK;
}

// Reads the counters and the time since count_begin into the context
// (mgk_ctx_last_loo_evals / mgk_ctx_last_loo_ms).
int count_end(mgk_ctx* c) {
    MGK_CHECK_CUDA(c, cudaEventRecord(c->ev_b, c->stream));
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(c->h_counter + 5, c->d_counter + 5, 2 * sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, c->stream));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->last_loo_evals[0] = (int64_t)c->h_counter[5];
    c->last_loo_evals[1] = (int64_t)c->h_counter[6];
    MGK_CHECK_CUDA(c, cudaEventElapsedTime(&c->last_loo_ms, c->ev_a, c->ev_b));
    return MGK_OK;
}

// den[input order] and logsum[0] = sum_j log(max(den_j, floor_v)).
int point_density(mgk_ctx* c, const mgk_index* idx, bool self, double* d_den, double floor_v, double* d_logsum) {
    cudaStream_t s = c->stream;
    const int64_t g = (idx->n + kPdQ - 1) / kPdQ;
    if (g == 0) {
        MGK_CHECK_CUDA(c, cudaMemsetAsync(d_logsum, 0, sizeof(double), s));
        return MGK_OK;
    }
    // bin rows split over enough CTAs to give every SM about 8 of them
    const int nsplit = (int)std::min<int64_t>(8, std::max<int64_t>(1, (8 * (int64_t)c->sm_count + g - 1) / g));
    const int64_t nbins = idx->varh ? idx->nbx * idx->nby : 0;
    const size_t b_part = sizeof(double) * (size_t)g, b_r2 = sizeof(float) * (size_t)std::max<int64_t>(nbins, 1);
    const size_t b_psum = sizeof(double) * (size_t)idx->n * (size_t)nsplit;
    double *part = nullptr, *psum = nullptr;
    float* r2 = nullptr;
    int st = mgk_alloc(c, (void**)&part, b_part);
    if (st) return st;
    if ((st = mgk_alloc(c, (void**)&psum, b_psum))) {
        mgk_free(c, part, b_part);
        return st;
    }
    if (idx->varh && (st = mgk_alloc(c, (void**)&r2, b_r2))) {
        mgk_free(c, part, b_part);
        mgk_free(c, psum, b_psum);
        return st;
    }
    const dim3 grid((unsigned)g, (unsigned)nsplit);
    if (idx->varh) {
        k_bin_reach2<<<(unsigned)((nbins + 255) / 256), 256, 0, s>>>(nbins, idx->bin_start, idx->pts, r2);
        k_point_density<true, false><<<grid, kPdQ, 0, s>>>(idx->n, idx->pts, idx->bin_start, idx->ox,
                                                           idx->oy, idx->side, idx->nbx, idx->nby, idx->reach,
                                                           idx->h2, r2, std::ldexp(1.0, -idx->qexp), psum,
                                                           pair_count(c));
    } else if (self) {
        k_point_density<false, true><<<grid, kPdQ, 0, s>>>(idx->n, idx->pts, idx->bin_start, idx->ox,
                                                           idx->oy, idx->side, idx->nbx, idx->nby, idx->reach,
                                                           idx->h2, nullptr, std::ldexp(1.0, -idx->qexp), psum,
                                                           pair_count(c));
    } else {
        k_point_density<false, false><<<grid, kPdQ, 0, s>>>(idx->n, idx->pts, idx->bin_start, idx->ox,
                                                            idx->oy, idx->side, idx->nbx, idx->nby, idx->reach,
                                                            idx->h2, nullptr, std::ldexp(1.0, -idx->qexp), psum,
                                                            pair_count(c));
    }
    k_pd_combine<<<(unsigned)g, kPdQ, 0, s>>>(idx->n, nsplit, psum, idx->perm, idx->varh, idx->h2, floor_v, d_den,
                                              part);
    k_sum_parts<<<1, 256, 0, s>>>(g, part, d_logsum);
    const cudaError_t e = cudaGetLastError();
    // pooled blocks: a later allocation of them is ordered on the same stream
    mgk_free(c, part, b_part);
    mgk_free(c, psum, b_psum);
    if (r2) mgk_free(c, r2, b_r2);
    if (e != cudaSuccess) return mgk_cuda_fail(c, e, "k_point_density");
    MGK_COUNT_LAUNCH(c, idx->varh ? 4 : 3);
    return MGK_OK;
}

// Pilot densities by bandwidth.  The search evaluates the likelihood at
// (h, alpha) pairs that share h (the centre and its two alpha neighbours),
// and the pilot density with its log sum (steps 1-3 up to the geometric
// mean) depends on h alone, so it is kept for the last few h.
struct PilotCache {
    static constexpr int kEntries = 6;
    mgk_ctx* c = nullptr;
    int64_t n = 0;
    uint32_t hbits[kEntries] = {};
    double* buf[kEntries] = {};  // den0[max(n, 1)], then the log sum
    uint64_t last[kEntries] = {};
    uint64_t tick = 0;
    size_t bytes() const { return sizeof(double) * (size_t)(std::max<int64_t>(n, 1) + 1); }
    ~PilotCache() {
        for (int i = 0; i < kEntries; i++)
            if (buf[i]) mgk_free(c, buf[i], bytes());
    }
};

// Steps 1-3 up to the geometric mean for bandwidth h: den0 (input order) and
// its log sum, computed or taken from the cache.
int pilot_density(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h, PilotCache& pc, double** den0) {
    uint32_t hb;
    memcpy(&hb, &h, sizeof(hb));
    int slot = -1;
    for (int i = 0; i < PilotCache::kEntries; i++)
        if (pc.buf[i] && pc.hbits[i] == hb) slot = i;
    if (slot >= 0) {
        pc.last[slot] = ++pc.tick;
        *den0 = pc.buf[slot];
        return MGK_OK;
    }
    for (int i = 0; i < PilotCache::kEntries; i++)  // a free entry, else the least recently used
        if (slot < 0 || !pc.buf[i] || (pc.buf[slot] && pc.last[i] < pc.last[slot])) slot = i;
    int st;
    if (!pc.buf[slot] && (st = mgk_alloc(c, (void**)&pc.buf[slot], pc.bytes()))) return st;
    pc.hbits[slot] = hb;
    pc.last[slot] = ++pc.tick;
    double* den = pc.buf[slot];
    if (r) st = mgk_launch_edge_weights(c, p->n, p->x, p->y, nullptr, h, p->dist2, r, p->ew, edge_count(c));
    else st = mgk_edge_weights_unit(c, p);
    if (st == MGK_OK) {
        p->has_ew = true;
        mgk_index* idx = nullptr;
        if ((st = mgk_index_build(c, p, h, 0.0f, &idx)) == MGK_OK) {  // h > 0: fixed-h index
            st = point_density(c, idx, true, den, 0.0, den + std::max<int64_t>(p->n, 1));
            mgk_index_destroy(idx);
        }
    }
    if (st) {
        pc.hbits[slot] = 0;  // not a valid entry
        mgk_free(c, pc.buf[slot], pc.bytes());
        pc.buf[slot] = nullptr;
        return st;
    }
    *den0 = den;
    return MGK_OK;
}

// Steps 1-3: the pilot density at h and hs = h (den0 / gml)^alpha into p->h.
int pilot_bandwidths(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h, float alpha, PilotCache& pc) {
    double* den0 = nullptr;
    int st = pilot_density(c, p, r, h, pc, &den0);
    if (st == MGK_OK && p->n > 0) {
        k_adaptive_h<<<(unsigned)((p->n + 255) / 256), 256, 0, c->stream>>>(p->n, den0, den0 + p->n, h, alpha, p->h);
        MGK_COUNT_LAUNCH(c, 1);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = mgk_cuda_fail(c, e, "adaptive bandwidths");
    }
    return st;
}

// LogLikelihood(h, alpha): steps 1-6.
int loglik_adaptive(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h, float alpha, double* d_den,
                    double* d_scal, double* logl, PilotCache& pc) {
    int st = pilot_bandwidths(c, p, r, h, alpha, pc);
    if (st) return st;
    if (r && (st = mgk_launch_edge_weights(c, p->n, p->x, p->y, p->h, 0.0f, p->dist2, r, p->ew, edge_count(c))))
        return st;
    // per-point h; bins of 0.75 h (the geometric mean of hs is h), not of the
    // widest h, so that the per-bin reach can cut the window down
    mgk_index* idx = nullptr;
    if ((st = mgk_index_build(c, p, 0.0f, 0.75f * h, &idx))) return st;
    st = point_density(c, idx, false, d_den, (double)MGK_EPS_DENSITY_F, d_scal + 1);
    mgk_index_destroy(idx);
    if (st) return st;
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(c->h_sum, d_scal + 1, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    *logl = c->h_sum[0];
    return MGK_OK;
}

// The search writes the bandwidths into p->h.  Points that wrap caller
// memory get a buffer of their own, so the caller's array is never written.
int ensure_h(mgk_ctx* c, mgk_points* p) {
    if (p->h && (p->owns_xywh || p->owns_h)) return MGK_OK;
    float* h = nullptr;
    const int st = mgk_alloc(c, (void**)&h, sizeof(float) * (size_t)std::max<int64_t>(p->n, 1));
    if (st) return st;
    p->h = h;
    if (!p->owns_xywh) p->owns_h = true;
    return MGK_OK;
}

}  // namespace

extern "C" {

int mgk_loglik_adaptive(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h, float alpha, double* logl) {
    if (!c || !p || !logl || !(h > 0.0f)) return mgk_fail(c, MGK_ERR_INVALID, "loglik_adaptive: bad arguments");
    if (r && !p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "loglik_adaptive: run mgk_boundary_dist first");
    if (r && std::isfinite(p->dist2_cap))  // the adaptive bandwidths are not known in advance
        return mgk_fail(c, MGK_ERR_INVALID, "loglik_adaptive: needs the exact boundary distances of mgk_boundary_dist");
    int st;
    if ((st = ensure_h(c, p))) return st;
    double *d_den = nullptr, *d_scal = nullptr;
    const size_t bd = sizeof(double) * (size_t)std::max<int64_t>(p->n, 1);
    if ((st = mgk_alloc(c, (void**)&d_den, bd))) return st;
    if ((st = mgk_alloc(c, (void**)&d_scal, 2 * sizeof(double)))) {
        mgk_free(c, d_den, bd);
        return st;
    }
    {
        PilotCache pc;
        pc.c = c;
        pc.n = p->n;
        st = count_begin(c);
        if (st == MGK_OK) st = loglik_adaptive(c, p, r, h, alpha, d_den, d_scal, logl, pc);
        if (st == MGK_OK) st = count_end(c);
    }
    mgk_free(c, d_den, bd);
    mgk_free(c, d_scal, 2 * sizeof(double));
    return st;
}

int mgk_adaptive_bandwidths(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h0, float* h_opt,
                            float* alpha_opt, double* lmax, int* iterations, float* hs_out) {
    if (!c || !p || !(h0 > 0.0f)) return mgk_fail(c, MGK_ERR_INVALID, "adaptive_bandwidths: bad arguments");
    if (r && !p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "adaptive_bandwidths: run mgk_boundary_dist first");
    if (r && std::isfinite(p->dist2_cap))  // the adaptive bandwidths are not known in advance
        return mgk_fail(c, MGK_ERR_INVALID, "adaptive_bandwidths: needs the exact boundary distances of mgk_boundary_dist");
    int st;
    if ((st = ensure_h(c, p))) return st;
    double *d_den = nullptr, *d_scal = nullptr;
    const size_t bd = sizeof(double) * (size_t)std::max<int64_t>(p->n, 1);
    if ((st = mgk_alloc(c, (void**)&d_den, bd))) return st;
    if ((st = mgk_alloc(c, (void**)&d_scal, 2 * sizeof(double)))) {
        mgk_free(c, d_den, bd);
        return st;
    }
    // hooke_jeeves (kde_cuda_kdtr_tiled.cu:3726-3785): float steps, five likelihoods
    float alpha0 = -0.5f;
    float stepH = h0 / 10;
    float stepA = 0.1f;
    // the likelihoods are kept as floats, the type of the reference's Ls array,
    // so that ties and near-ties compare as they do there
    float L[5] = {0, 0, 0, 0, 0};
    PilotCache pc;
    pc.c = c;
    pc.n = p->n;
    auto ll = [&](float h, float a, float* out) {
        double v = 0.0;
        const int s1 = loglik_adaptive(c, p, r, h, a, d_den, d_scal, &v, pc);
        *out = (float)v;
        return s1;
    };
    // hj_likelihood (:3677-3720): the centre and the neighbours the last move did not keep
    auto around = [&](int last) {
        int s2 = MGK_OK;
        if (s2 == MGK_OK && last == -1) s2 = ll(h0, alpha0, &L[0]);
        if (s2 == MGK_OK && last != 2) s2 = ll(h0 - stepH, alpha0, &L[1]);
        if (s2 == MGK_OK && last != 1) s2 = ll(h0 + stepH, alpha0, &L[2]);
        if (s2 == MGK_OK && last != 4) s2 = ll(h0, alpha0 + stepA, &L[3]);
        if (s2 == MGK_OK && last != 3) s2 = ll(h0, alpha0 - stepA, &L[4]);
        return s2;
    };
    st = count_begin(c);
    if (st == MGK_OK) st = around(-1);
    float Lm = L[0];
    const float sH = stepH / 10, sA = stepA / 10;
    int it = 0;
    while (st == MGK_OK && (stepH > sH || stepA > sA) && (h0 - stepH > 0) && it <= 30) {  // MAX_NUM_ITERATIONS
        int dmax = 0;
        for (int i = 0; i < 5; i++)
            if (L[i] > Lm) {
                Lm = L[i];
                dmax = i;
            }
        if (dmax == 0) {
            stepH = stepH / 2;
            stepA = stepA / 2;
        } else {
            // the reference's moves and its bookkeeping of the kept likelihoods
            // (:3750-3778), the move to +stepA included
            if (dmax == 1) {
                h0 = h0 - stepH;
                L[2] = L[0];
                L[0] = L[1];
            }
            if (dmax == 2) {
                h0 = h0 + stepH;
                L[1] = L[0];
                L[0] = L[2];
            }
            if (dmax == 3) {
                alpha0 = alpha0 + stepA;
                L[3] = L[0];
                L[0] = L[4];
            }
            if (dmax == 4) {
                alpha0 = alpha0 - stepA;
                L[3] = L[0];
                L[0] = L[4];
            }
        }
        st = around(dmax);
        it++;
    }
    // final bandwidths at the optimum (main :566-572)
    if (st == MGK_OK) st = pilot_bandwidths(c, p, r, h0, alpha0, pc);
    if (st == MGK_OK && hs_out && p->n > 0) {
        const cudaError_t e = cudaMemcpyAsync(hs_out, p->h, sizeof(float) * (size_t)p->n, cudaMemcpyDeviceToHost,
                                              c->stream);
        if (e != cudaSuccess) st = mgk_cuda_fail(c, e, "adaptive bandwidths download");
    }
    if (st == MGK_OK) st = count_end(c);
    mgk_free(c, d_den, bd);
    mgk_free(c, d_scal, 2 * sizeof(double));
    if (st) return st;
    p->has_ew = false;  // the weights left behind belong to the fixed h0; recompute at hs
    if (h_opt) *h_opt = h0;
    if (alpha_opt) *alpha_opt = alpha0;
    if (lmax) *lmax = Lm;
    if (iterations) *iterations = it;
    return MGK_OK;
}

}  // extern "C"
