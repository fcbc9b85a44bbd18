// C ABI of libmgk (include/mgk.h): contexts, device-resident objects, and the
// host-side sequencing of the path (the GPU section of the reference's
// main(), kde_cuda_kdtr_tiled.cu:877-1521, for one GPU).
#include <cudaTypedefs.h>

#include <immintrin.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "mgk_internal.cuh"

// ---------------------------------------------------------------- helpers --
int mgk_fail(mgk_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

int mgk_cuda_fail(mgk_ctx* ctx, cudaError_t e, const char* what) {
    (void)cudaGetLastError();  // clear sticky-less errors
    return mgk_fail(ctx, e == cudaErrorMemoryAllocation ? MGK_ERR_BUDGET : MGK_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
}

// Device memory of a context is cached: a freed block goes back to a pool
// keyed by its size class and is handed out again to the next request of that
// class, so a step that allocates and frees the same scratch every call
// (index build, tile plans) does not pay cudaMalloc/cudaFree each time.  All
// work of a context is ordered on its stream, so a block reused by a later
// launch is only touched after the earlier launches that used it.  Pooled
// bytes count against the HBM budget; when a request would exceed it the pool
// is released first.
static size_t size_class(size_t bytes) {
    if (bytes <= 256) return 256;
    if (bytes <= (1u << 20)) {
        size_t c = 256;
        while (c < bytes) c <<= 1;
        return c;
    }
    const size_t g = 2u << 20;
    return (bytes + g - 1) / g * g;
}

static void release_pool(mgk_ctx* ctx) {
    for (auto& kv : ctx->pool) {
        cudaFree(kv.second);
        ctx->in_use -= std::min<uint64_t>(ctx->in_use, kv.first);
    }
    ctx->pool.clear();
}

int mgk_alloc(mgk_ctx* ctx, void** p, size_t bytes) {
    *p = nullptr;
    const size_t cls = size_class(bytes ? bytes : 16);
    auto it = ctx->pool.find(cls);
    if (it != ctx->pool.end()) {
        *p = it->second;
        ctx->pool.erase(it);
        return MGK_OK;
    }
    if (ctx->in_use + cls > ctx->budget && !ctx->pool.empty()) release_pool(ctx);
    if (ctx->in_use + cls > ctx->budget)
        return mgk_fail(ctx, MGK_ERR_BUDGET,
                        "HBM budget exceeded: need " + std::to_string(cls) + " B, in use " +
                            std::to_string(ctx->in_use.load()) + " of " + std::to_string(ctx->budget));
    cudaError_t e = cudaMalloc(p, cls);
    if (e == cudaErrorMemoryAllocation && !ctx->pool.empty()) {
        (void)cudaGetLastError();
        release_pool(ctx);
        e = cudaMalloc(p, cls);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return mgk_cuda_fail(ctx, e, "cudaMalloc");
    }
    ctx->in_use += cls;
    return MGK_OK;
}

int mgk_host_stage_slot(mgk_ctx* c, int slot, size_t bytes, void** host, void** dev) {
    if (slot < 0 || slot >= mgk_ctx::kStageSlots) return mgk_fail(c, MGK_ERR_INVALID, "staging slot out of range");
    if (bytes > c->h_stage_bytes[slot]) {
        if (c->h_stage[slot]) cudaFreeHost(c->h_stage[slot]);
        c->h_stage[slot] = nullptr;
        c->d_stage[slot] = nullptr;
        c->h_stage_bytes[slot] = 0;
        const size_t want = std::max<size_t>(bytes + bytes / 4, 1 << 16);
        cudaError_t e = cudaHostAlloc(&c->h_stage[slot], want, cudaHostAllocMapped);
        if (e != cudaSuccess) {
            c->h_stage[slot] = nullptr;
            return mgk_cuda_fail(c, e, "mapped page-locked staging");
        }
        e = cudaHostGetDevicePointer(&c->d_stage[slot], c->h_stage[slot], 0);
        if (e != cudaSuccess) {
            cudaFreeHost(c->h_stage[slot]);
            c->h_stage[slot] = nullptr;
            return mgk_cuda_fail(c, e, "mapped page-locked staging address");
        }
        c->h_stage_bytes[slot] = want;
    }
    *host = c->h_stage[slot];
    *dev = c->d_stage[slot];
    return MGK_OK;
}

int mgk_host_stage(mgk_ctx* c, size_t bytes, void** host, void** dev) {
    return mgk_host_stage_slot(c, 0, bytes, host, dev);
}

void mgk_free(mgk_ctx* ctx, void* p, size_t bytes) {
    if (!p) return;
    ctx->pool.emplace(size_class(bytes ? bytes : 16), p);
}

extern "C" {

const char* mgk_status_string(int status) {
    switch (status) {
        case MGK_OK: return "ok";
        case MGK_ERR_INVALID: return "invalid argument";
        case MGK_ERR_CUDA: return "CUDA error";
        case MGK_ERR_BUDGET: return "HBM budget exceeded";
        case MGK_ERR_NO_DEVICE: return "no suitable CUDA device";
        case MGK_ERR_TIMEOUT: return "device wait timed out";
        case MGK_ERR_IO: return "I/O error";
        default: return "unknown status";
    }
}

// ---------------------------------------------------------------- context --
int mgk_ctx_create(int device, uint64_t hbm_budget_bytes, mgk_ctx** out) {
    if (!out) return MGK_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        (void)cudaGetLastError();
        return MGK_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return MGK_ERR_INVALID;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MGK_ERR_NO_DEVICE;
    if (prop.major != 10) return MGK_ERR_NO_DEVICE;  // built for sm_100a only
    if (cudaSetDevice(device) != cudaSuccess) return MGK_ERR_CUDA;
    mgk_ctx* c = new (std::nothrow) mgk_ctx();
    if (!c) return MGK_ERR_INVALID;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    c->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)fr;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return MGK_ERR_CUDA;
    }
    c->stream = c->own_stream;
    if (cudaMalloc(&c->d_counter, 8 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&c->d_sum, 256 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&c->h_counter, 8 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost(&c->h_sum, 256 * sizeof(double)) != cudaSuccess ||
        cudaEventCreate(&c->ev_a) != cudaSuccess || cudaEventCreate(&c->ev_b) != cudaSuccess) {
        mgk_ctx_destroy(c);
        return MGK_ERR_CUDA;
    }
    *out = c;
    return MGK_OK;
}

int mgk_ctx_destroy(mgk_ctx* c) {
    if (!c) return MGK_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    release_pool(c);
    if (c->d_counter) cudaFree(c->d_counter);
    if (c->d_sum) cudaFree(c->d_sum);
    if (c->h_counter) cudaFreeHost(c->h_counter);
    if (c->h_sum) cudaFreeHost(c->h_sum);
    for (int i = 0; i < mgk_ctx::kStageSlots; i++)
        if (c->h_stage[i]) cudaFreeHost(c->h_stage[i]);
    if (c->ev_a) cudaEventDestroy(c->ev_a);
    if (c->ev_b) cudaEventDestroy(c->ev_b);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return MGK_OK;
}

int mgk_ctx_set_stream(mgk_ctx* c, void* stream) {
    if (!c) return MGK_ERR_INVALID;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return MGK_OK;
}

int mgk_ctx_synchronize(mgk_ctx* c) {
    if (!c) return MGK_ERR_INVALID;
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    return MGK_OK;
}

const char* mgk_ctx_last_error(const mgk_ctx* c) { return c ? c->last_error.c_str() : "no context"; }

uint64_t mgk_ctx_bytes_in_use(const mgk_ctx* c) { return c ? c->in_use.load() : 0; }

uint64_t mgk_ctx_kernel_launches(const mgk_ctx* c) { return c ? c->launches : 0; }

float mgk_ctx_last_density_ms(const mgk_ctx* c) { return c ? c->last_density_ms : 0.0f; }
float mgk_ctx_last_loo_ms(const mgk_ctx* c) { return c ? c->last_loo_ms : 0.0f; }
int mgk_ctx_last_loo_evals(const mgk_ctx* c, int64_t* edge_evals, int64_t* loo_evals) {
    if (!c) return MGK_ERR_INVALID;
    if (edge_evals) *edge_evals = c->last_loo_evals[0];
    if (loo_evals) *loo_evals = c->last_loo_evals[1];
    return MGK_OK;
}

// ----------------------------------------------------------------- points --
static int points_alloc_results(mgk_ctx* c, mgk_points* p) {
    int st;
    if ((st = mgk_alloc(c, (void**)&p->dist2, sizeof(double) * std::max<int64_t>(p->n, 1)))) return st;
    if ((st = mgk_alloc(c, (void**)&p->ew, sizeof(float) * std::max<int64_t>(p->n, 1)))) return st;
    return MGK_OK;
}

int mgk_points_upload(mgk_ctx* c, int64_t n, const float* x, const float* y, const float* w, const float* h,
                      mgk_points** out) {
    if (!c || !out || n < 0 || (n > 0 && (!x || !y))) return mgk_fail(c, MGK_ERR_INVALID, "points_upload: bad arguments");
    if (n >= (int64_t)INT32_MAX) return mgk_fail(c, MGK_ERR_INVALID, "points_upload: at most 2^31-1 points");
    mgk_points* p = new (std::nothrow) mgk_points();
    if (!p) return MGK_ERR_INVALID;
    p->ctx = c;
    p->n = n;
    p->owns_xywh = true;
    const size_t b = sizeof(float) * (size_t)std::max<int64_t>(n, 1);
    int st = MGK_OK;
    if ((st = mgk_alloc(c, (void**)&p->x, b)) || (st = mgk_alloc(c, (void**)&p->y, b)) ||
        (w && (st = mgk_alloc(c, (void**)&p->w, b))) || (h && (st = mgk_alloc(c, (void**)&p->h, b))) ||
        (st = points_alloc_results(c, p))) {
        mgk_points_destroy(p);
        return st;
    }
    const size_t nb = sizeof(float) * (size_t)n;
    cudaStream_t s = c->stream;
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        if (e == cudaSuccess) e = cudaMemcpyAsync(p->x, x, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(p->y, y, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && w) e = cudaMemcpyAsync(p->w, w, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && h) e = cudaMemcpyAsync(p->h, h, nb, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host buffers may be pageable/temporary
    }
    if (e != cudaSuccess) {
        mgk_points_destroy(p);
        return mgk_cuda_fail(c, e, "points_upload");
    }
    *out = p;
    return MGK_OK;
}

int mgk_points_wrap(mgk_ctx* c, int64_t n, const float* d_x, const float* d_y, const float* d_w, const float* d_h,
                    mgk_points** out) {
    if (!c || !out || n < 0 || (n > 0 && (!d_x || !d_y))) return mgk_fail(c, MGK_ERR_INVALID, "points_wrap: bad arguments");
    if (n >= (int64_t)INT32_MAX) return mgk_fail(c, MGK_ERR_INVALID, "points_wrap: at most 2^31-1 points");
    mgk_points* p = new (std::nothrow) mgk_points();
    if (!p) return MGK_ERR_INVALID;
    p->ctx = c;
    p->n = n;
    p->owns_xywh = false;
    p->x = const_cast<float*>(d_x);
    p->y = const_cast<float*>(d_y);
    p->w = const_cast<float*>(d_w);
    p->h = const_cast<float*>(d_h);
    int st = points_alloc_results(c, p);
    if (st) {
        mgk_points_destroy(p);
        return st;
    }
    *out = p;
    return MGK_OK;
}

int64_t mgk_points_size(const mgk_points* p) { return p ? p->n : 0; }

int mgk_points_select(mgk_ctx* c, const mgk_points* src, double xlo, double xhi, double ylo, double yhi,
                      mgk_points** out) {
    if (!c || !src || !out || !(xlo <= xhi) || !(ylo <= yhi))
        return mgk_fail(c, MGK_ERR_INVALID, "points_select: bad arguments");
    *out = nullptr;
    const size_t bs = sizeof(unsigned) * (size_t)mgk_points_select_scratch(src->n);
    unsigned* scr = nullptr;
    int st = mgk_alloc(c, (void**)&scr, bs);
    if (st) return st;
    int64_t m = 0;
    st = mgk_launch_points_select(c, src, xlo, xhi, ylo, yhi, scr, &m, nullptr);
    mgk_points* p = nullptr;
    if (st == MGK_OK) {
        p = new (std::nothrow) mgk_points();
        if (!p) st = MGK_ERR_INVALID;
    }
    if (st == MGK_OK) {
        p->ctx = c;
        p->n = m;
        p->owns_xywh = true;
        const size_t b = sizeof(float) * (size_t)std::max<int64_t>(m, 1);
        if ((st = mgk_alloc(c, (void**)&p->x, b)) == MGK_OK && (st = mgk_alloc(c, (void**)&p->y, b)) == MGK_OK &&
            (!src->w || (st = mgk_alloc(c, (void**)&p->w, b)) == MGK_OK) &&
            (!src->h || (st = mgk_alloc(c, (void**)&p->h, b)) == MGK_OK))
            st = points_alloc_results(c, p);
        if (st == MGK_OK) st = mgk_launch_points_select(c, src, xlo, xhi, ylo, yhi, scr, &m, p);
    }
    mgk_free(c, scr, bs);  // stream-ordered reuse: later users run after the scatter
    if (st) {
        mgk_points_destroy(p);
        return st;
    }
    *out = p;
    return MGK_OK;
}

int mgk_points_destroy(mgk_points* p) {
    if (!p) return MGK_OK;
    mgk_ctx* c = p->ctx;
    const size_t b = sizeof(float) * (size_t)std::max<int64_t>(p->n, 1);
    if (p->owns_xywh) {
        mgk_free(c, p->x, b);
        mgk_free(c, p->y, b);
        mgk_free(c, p->w, b);
        mgk_free(c, p->h, b);
    } else if (p->owns_h) {
        mgk_free(c, p->h, b);
    }
    mgk_free(c, p->dist2, sizeof(double) * (size_t)std::max<int64_t>(p->n, 1));
    mgk_free(c, p->ew, b);
    delete p;
    return MGK_OK;
}

int mgk_points_device_arrays(const mgk_points* p, const float** x, const float** y, const float** w,
                             const float** h, const double** dist2, const float** ew) {
    if (!p) return MGK_ERR_INVALID;
    if (x) *x = p->x;
    if (y) *y = p->y;
    if (w) *w = p->w;
    if (h) *h = p->h;
    if (dist2) *dist2 = p->has_dist2 ? p->dist2 : nullptr;
    if (ew) *ew = p->has_ew ? p->ew : nullptr;
    return MGK_OK;
}

int mgk_points_download(mgk_points* p, double* dist2, float* ew) {
    if (!p) return MGK_ERR_INVALID;
    mgk_ctx* c = p->ctx;
    cudaStream_t s = c->stream;
    if (dist2) {
        if (!p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "points_download: no distances computed");
        MGK_CHECK_CUDA(c, cudaMemcpyAsync(dist2, p->dist2, sizeof(double) * p->n, cudaMemcpyDeviceToHost, s));
    }
    if (ew) {
        if (!p->has_ew) return mgk_fail(c, MGK_ERR_INVALID, "points_download: no edge weights computed");
        MGK_CHECK_CUDA(c, cudaMemcpyAsync(ew, p->ew, sizeof(float) * p->n, cudaMemcpyDeviceToHost, s));
    }
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(s));
    return MGK_OK;
}

// ----------------------------------------------------------------- raster --
static bool grid_ok(const mgk_grid* g) {
    return g && g->ncols > 0 && g->nrows > 0 && g->cs > 0.0f && std::isfinite(g->cs) && std::isfinite(g->xll) &&
           std::isfinite(g->yll);
}

int mgk_raster_upload(mgk_ctx* c, const mgk_grid* g, const float* mask, mgk_raster** out) {
    if (!c || !out || !grid_ok(g) || !mask) return mgk_fail(c, MGK_ERR_INVALID, "raster_upload: bad arguments");
    mgk_raster* r = new (std::nothrow) mgk_raster();
    if (!r) return MGK_ERR_INVALID;
    r->ctx = c;
    r->g = *g;
    r->owns = true;
    const size_t b = sizeof(float) * (size_t)g->ncols * (size_t)g->nrows;
    int st = mgk_alloc(c, (void**)&r->mask, b);
    if (st) {
        delete r;
        return st;
    }
    cudaError_t e = cudaMemcpyAsync(r->mask, mask, b, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        mgk_raster_destroy(r);
        return mgk_cuda_fail(c, e, "raster_upload");
    }
    *out = r;
    return MGK_OK;
}

int mgk_raster_wrap(mgk_ctx* c, const mgk_grid* g, const float* d_mask, mgk_raster** out) {
    if (!c || !out || !grid_ok(g) || !d_mask) return mgk_fail(c, MGK_ERR_INVALID, "raster_wrap: bad arguments");
    mgk_raster* r = new (std::nothrow) mgk_raster();
    if (!r) return MGK_ERR_INVALID;
    r->ctx = c;
    r->g = *g;
    r->owns = false;
    r->mask = const_cast<float*>(d_mask);
    *out = r;
    return MGK_OK;
}

int mgk_raster_destroy(mgk_raster* r) {
    if (!r) return MGK_OK;
    mgk_ctx* c = r->ctx;
    const size_t ncell = (size_t)r->g.ncols * (size_t)r->g.nrows;
    if (r->owns) mgk_free(c, r->mask, sizeof(float) * ncell);
    mgk_free(c, r->boundary, ncell);
    mgk_free(c, r->bcells, sizeof(float2) * (size_t)std::max<int64_t>(r->nb, 1));
    mgk_free(c, r->bstart, sizeof(int) * (size_t)(r->nbins + 1));
    mgk_free(c, r->bnear, sizeof(int) * (size_t)(r->nbins + 1));
    mgk_free(c, r->bub, sizeof(double) * (size_t)r->nbins);
    mgk_free(c, r->cstart, sizeof(int) * (size_t)(r->nbins + 1));
    mgk_free(c, r->cand, sizeof(float2) * (size_t)std::max<int64_t>(r->ncand, 1));
    mgk_free(c, r->run_start, sizeof(int64_t) * (size_t)(r->g.nrows + 1));
    mgk_free(c, r->runs, sizeof(int2) * (size_t)std::max<int64_t>(r->nruns, 1));
    delete r;
    return MGK_OK;
}

// --------------------------------------------------------------- boundary --
int mgk_mark_boundary(mgk_ctx* c, mgk_raster* r, int64_t* n_boundary) {
    if (!c || !r) return mgk_fail(c, MGK_ERR_INVALID, "mark_boundary: bad arguments");
    int st = mgk_launch_mark_boundary(c, r);
    if (st) return st;
    if (n_boundary) *n_boundary = r->nb;
    return MGK_OK;
}

int mgk_raster_boundary_download(mgk_raster* r, uint8_t* out) {
    if (!r || !out) return MGK_ERR_INVALID;
    mgk_ctx* c = r->ctx;
    if (!r->marked) return mgk_fail(c, MGK_ERR_INVALID, "boundary not marked");
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(out, r->boundary, (size_t)r->g.ncols * r->g.nrows, cudaMemcpyDeviceToHost, c->stream));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    return MGK_OK;
}

static int boundary_dist(mgk_ctx* c, mgk_points* p, mgk_raster* r, double cap) {
    int st;
    if (!r->marked && (st = mgk_launch_mark_boundary(c, r))) return st;
    if ((st = mgk_launch_dist2(c, p, r, cap))) return st;
    p->has_dist2 = true;
    p->dist2_cap = cap;
    return MGK_OK;
}

int mgk_boundary_dist(mgk_ctx* c, mgk_points* p, mgk_raster* r) {
    if (!c || !p || !r) return mgk_fail(c, MGK_ERR_INVALID, "boundary_dist: bad arguments");
    return boundary_dist(c, p, r, INFINITY);
}

int mgk_boundary_dist_within(mgk_ctx* c, mgk_points* p, mgk_raster* r, double reach) {
    if (!c || !p || !r || !(reach > 0.0)) return mgk_fail(c, MGK_ERR_INVALID, "boundary_dist_within: bad arguments");
    return boundary_dist(c, p, r, reach);
}

// The edge-weight short-circuit (weight 1 when dist2 >= 9 h^2, h^2 a float
// product) decides exactly from distances that are exact up to dist2_cap
// only if 9 h^2 <= dist2_cap^2 for every bandwidth used.
static bool cap_covers(const mgk_points* p, float hmax) {
    if (!std::isfinite(p->dist2_cap)) return true;
    return 9.0 * (double)(hmax * hmax) <= p->dist2_cap * p->dist2_cap;
}

__global__ static void k_max_h(int64_t n, const float* __restrict__ h, unsigned* out) {
    unsigned m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fmaxf(h[i], 0.0f)));  // non-negative floats order as their bits
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Largest per-point bandwidth (device reduction, one read back).
static int points_hmax(mgk_ctx* c, const mgk_points* p, float* out) {
    unsigned* d = reinterpret_cast<unsigned*>(c->d_counter);
    MGK_CHECK_CUDA(c, cudaMemsetAsync(d, 0, sizeof(unsigned), c->stream));
    if (p->n) k_max_h<<<(unsigned)std::min<int64_t>((p->n + 255) / 256, 4 * c->sm_count), 256, 0, c->stream>>>(
        p->n, p->h, d);
    MGK_CHECK_LAUNCH(c, "k_max_h");
    unsigned v = 0;
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(&v, d, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    memcpy(out, &v, sizeof(float));
    return MGK_OK;
}

// ------------------------------------------------------------ edge weights --
static int fetch_counter(mgk_ctx* c, int64_t* out) {
    MGK_CHECK_CUDA(c, cudaMemcpyAsync(c->h_counter, c->d_counter, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                      c->stream));
    MGK_CHECK_CUDA(c, cudaStreamSynchronize(c->stream));
    *out = (int64_t)c->h_counter[0];
    return MGK_OK;
}

int mgk_edge_weights(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h, int64_t* evals) {
    if (!c || !p || !r) return mgk_fail(c, MGK_ERR_INVALID, "edge_weights: bad arguments");
    if (!p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "edge_weights: run mgk_boundary_dist first");
    if (h <= 0.0f && !p->h) return mgk_fail(c, MGK_ERR_INVALID, "edge_weights: no bandwidth");
    float hmax = h;
    if (h <= 0.0f && std::isfinite(p->dist2_cap)) {
        int st = points_hmax(c, p, &hmax);
        if (st) return st;
    }
    if (!cap_covers(p, hmax))
        return mgk_fail(c, MGK_ERR_INVALID, "edge_weights: the boundary distances are exact only within " +
                                                std::to_string(p->dist2_cap) + " (< 3h); use a larger reach");
    if (evals) MGK_CHECK_CUDA(c, cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned long long), c->stream));
    int st = mgk_launch_edge_weights(c, p->n, p->x, p->y, h > 0.0f ? nullptr : p->h, h, p->dist2, r, p->ew,
                                     evals ? c->d_counter : nullptr);
    if (st) return st;
    p->has_ew = true;
    if (evals) return fetch_counter(c, evals);
    return MGK_OK;
}

__global__ static void k_fill1(int64_t n, float* a) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = 1.0f;
}

int mgk_edge_weights_unit(mgk_ctx* c, mgk_points* p) {
    if (!c || !p) return MGK_ERR_INVALID;
    if (p->n) k_fill1<<<(unsigned)((p->n + 255) / 256), 256, 0, c->stream>>>(p->n, p->ew);
    MGK_CHECK_LAUNCH(c, "k_fill1");
    if (p->n) MGK_COUNT_LAUNCH(c, 1);
    p->has_ew = true;
    return MGK_OK;
}

// ------------------------------------------------------------------ index --
int mgk_index_build(mgk_ctx* c, const mgk_points* p, float h, float bin_size, mgk_index** out) {
    if (!c || !p || !out) return mgk_fail(c, MGK_ERR_INVALID, "index_build: bad arguments");
    mgk_index* idx = new (std::nothrow) mgk_index();
    if (!idx) return MGK_ERR_INVALID;
    int st = mgk_launch_index_build(c, p, h, bin_size, idx);
    if (st) {
        mgk_index_destroy(idx);
        return st;
    }
    *out = idx;
    return MGK_OK;
}

int mgk_index_destroy(mgk_index* idx) {
    if (!idx) return MGK_OK;
    mgk_ctx* c = idx->ctx;
    if (c) {
        const size_t n1 = (size_t)std::max<int64_t>(idx->n, 1);
        mgk_free(c, idx->bin_start, sizeof(int32_t) * (size_t)(idx->nbx * idx->nby + 1));
        mgk_free(c, idx->pts, sizeof(MgkPt) * n1);
        mgk_free(c, idx->perm, sizeof(int32_t) * n1);
    }
    delete idx;
    return MGK_OK;
}

// ---------------------------------------------------------------- density --
static int density_common(mgk_ctx* c, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                          int64_t nr, int64_t nc, const float* d_mask, float* d_out, int64_t* evals, bool fp64) {
    if (!c || !idx || !grid_ok(g) || !d_out) return mgk_fail(c, MGK_ERR_INVALID, "density_tile: bad arguments");
    if (row0 < 0 || col0 < 0 || nr < 0 || nc < 0 || row0 + nr > g->nrows || col0 + nc > g->ncols)
        return mgk_fail(c, MGK_ERR_INVALID, "density_tile: tile outside the raster");
    if (evals) MGK_CHECK_CUDA(c, cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned long long), c->stream));
    int st = mgk_launch_density(c, idx, g, row0, col0, nr, nc, d_mask, d_out, evals ? c->d_counter : nullptr, fp64);
    if (st) return st;
    if (evals) return fetch_counter(c, evals);
    return MGK_OK;
}

int mgk_density_tile(mgk_ctx* c, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0, int64_t nr,
                     int64_t nc, const float* d_mask, float* d_out, int64_t* evals) {
    return density_common(c, idx, g, row0, col0, nr, nc, d_mask, d_out, evals, false);
}

int mgk_density_tile_fp64(mgk_ctx* c, const mgk_index* idx, const mgk_grid* g, int64_t row0, int64_t col0,
                          int64_t nr, int64_t nc, const float* d_mask, float* d_out, int64_t* evals) {
    if (evals) *evals = -1;  // the FP64 form does not count
    return density_common(c, idx, g, row0, col0, nr, nc, d_mask, d_out, nullptr, true);
}

int mgk_density_tiles(mgk_ctx* c, int njobs, const mgk_tile_job* jobs, int64_t* evals) {
    if (!c || njobs < 0 || (njobs > 0 && !jobs)) return mgk_fail(c, MGK_ERR_INVALID, "density_tiles: bad arguments");
    for (int j = 0; j < njobs; j++) {
        const mgk_tile_job& J = jobs[j];
        if (!J.index || !grid_ok(&J.grid) || !J.d_out) return mgk_fail(c, MGK_ERR_INVALID, "density_tiles: bad job");
        if (J.row0 < 0 || J.col0 < 0 || J.nrows < 0 || J.ncols < 0 || J.row0 + J.nrows > J.grid.nrows ||
            J.col0 + J.ncols > J.grid.ncols)
            return mgk_fail(c, MGK_ERR_INVALID, "density_tiles: tile outside its raster");
    }
    unsigned long long* d_ev = nullptr;
    const size_t bev = sizeof(unsigned long long) * (size_t)std::max(njobs, 1);
    int st;
    if (evals) {
        if ((st = mgk_alloc(c, (void**)&d_ev, bev))) return st;
        MGK_CHECK_CUDA(c, cudaMemsetAsync(d_ev, 0, bev, c->stream));
    }
    st = mgk_launch_density_jobs(c, njobs, jobs, d_ev);
    if (st == MGK_OK && evals) {
        std::vector<unsigned long long> h(njobs);
        cudaError_t e = cudaMemcpyAsync(h.data(), d_ev, sizeof(unsigned long long) * njobs, cudaMemcpyDeviceToHost,
                                        c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) st = mgk_cuda_fail(c, e, "density_tiles evals");
        for (int j = 0; j < njobs && st == MGK_OK; j++) evals[j] = (int64_t)h[j];
    }
    mgk_free(c, d_ev, bev);
    return st;
}

// ------------------------------------------------------------ bandwidths --
float mgk_rule_of_thumb(int64_t n, const float* x, const float* y, const float* w) {
    // MeanCenter (float accumulators), StandardDistance2 (double), BandWidth2,
    // kde_cuda_kdtr_tiled.cu:64-68, 1563-1595.  Host code built for baseline
    // x86-64 (no FMA instructions), so each operation rounds on its own as in
    // the reference.
    float sum_x = 0.0f, sum_y = 0.0f, sum_w = 0.0f;
    for (int64_t p = 0; p < n; p++) {
        const float wp = w ? w[p] : 1.0f;
        sum_w += wp;
        sum_x += wp * x[p];
        sum_y += wp * y[p];
    }
    const float mx = sum_x / sum_w, my = sum_y / sum_w;
    double s2 = 0.0, sw = 0.0;
    for (int64_t p = 0; p < n; p++) {
        const float wp = w ? w[p] : 1.0f;
        sw += wp;
        const double dx = (double)(x[p] - mx);
        const double dy = (double)(y[p] - my);
        s2 += wp * (dx * dx + dy * dy);
    }
    const double d2 = s2 / sw;
    const unsigned int three_n = 3u * (unsigned int)n;
    const double bw2 = (double)sqrtf(2.0f / (float)three_n) * d2;
    return sqrtf((float)bw2);
}

// evaluates logL at each h; the index over the points (unit edge weights) is shared
static int check_bandwidths(mgk_ctx* c, const float* hs, int nh, float* lo, float* hi) {
    *lo = FLT_MAX;
    *hi = 0.0f;
    for (int k = 0; k < nh; k++) {
        if (!(hs[k] > 0.0f) || !std::isfinite(hs[k])) return mgk_fail(c, MGK_ERR_INVALID, "loo: bandwidths must be positive");
        *lo = std::min(*lo, hs[k]);
        *hi = std::max(*hi, hs[k]);
    }
    return MGK_OK;
}

int mgk_loo_loglik_batch(mgk_ctx* c, mgk_points* p, const mgk_raster* r, const float* h_grid, int nh, double* logl,
                         int* argmax) {
    if (!c || !p || !h_grid || nh <= 0 || !logl) return mgk_fail(c, MGK_ERR_INVALID, "loo_loglik_batch: bad arguments");
    if (r && !p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "loo: run mgk_boundary_dist first");
    float lo, hi;
    int st = check_bandwidths(c, h_grid, nh, &lo, &hi);
    if (st) return st;
    if (r && !cap_covers(p, hi))
        return mgk_fail(c, MGK_ERR_INVALID, "loo: the boundary distances are exact only within " +
                                                std::to_string(p->dist2_cap) + ", less than 3 h_max");
    mgk_loo_batch* B = nullptr;  // runs once: no graph
    if ((st = mgk_loo_batch_create_share(c, p, r, lo, hi, nh, 0, 1, nullptr, 0, &B, false))) return st;
    st = mgk_loo_batch_run(B, h_grid, logl, argmax, nullptr, nullptr);
    mgk_loo_batch_destroy(B);
    return st;
}

// ---------------------------------------------- multi-GPU bandwidth selection --
static inline int64_t share_chunk(int64_t n, int nparts) { return (n + nparts - 1) / nparts; }

int mgk_loo_share_edge_weights(mgk_ctx* c, mgk_points* p, const mgk_raster* r, const float* h_grid, int nh,
                               int part, int nparts, float* d_ew_all, int64_t* evals) {
    if (!c || !p || !r || !h_grid || nh <= 0 || !d_ew_all || nparts <= 0 || part < 0 || part >= nparts)
        return mgk_fail(c, MGK_ERR_INVALID, "loo_share_edge_weights: bad arguments");
    if (!p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "loo: run mgk_boundary_dist first");
    float lo, hi;
    int st = check_bandwidths(c, h_grid, nh, &lo, &hi);
    if (st) return st;
    if (!cap_covers(p, hi))
        return mgk_fail(c, MGK_ERR_INVALID, "loo: the boundary distances are exact only within " +
                                                std::to_string(p->dist2_cap) + ", less than 3 h_max");
    const int64_t ch = share_chunk(p->n, nparts);
    const int64_t p0 = std::min<int64_t>(p->n, (int64_t)part * ch), p1 = std::min<int64_t>(p->n, p0 + ch);
    float* d_h = nullptr;
    if ((st = mgk_alloc(c, (void**)&d_h, sizeof(float) * nh))) return st;
    cudaError_t ce = cudaMemcpyAsync(d_h, h_grid, sizeof(float) * nh, cudaMemcpyHostToDevice, c->stream);
    if (ce == cudaSuccess && evals) ce = cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned long long), c->stream);
    if (ce != cudaSuccess) st = mgk_cuda_fail(c, ce, "loo_share_edge_weights");
    if (st == MGK_OK && p1 > p0)
        st = mgk_launch_edge_weights_multi(c, p1 - p0, p->x + p0, p->y + p0, nullptr, 0.0f, d_h, nh, p->dist2 + p0,
                                           r, d_ew_all + (int64_t)part * nh * ch, ch,
                                           evals ? c->d_counter : nullptr);
    // the host copy of h_grid above is pageable: it has been staged before
    // the call returned, so the buffer can go back to the pool (stream order)
    mgk_free(c, d_h, sizeof(float) * nh);
    if (st) return st;
    if (evals) return fetch_counter(c, evals);
    return MGK_OK;
}

int mgk_loo_share_loglik(mgk_ctx* c, mgk_points* p, const float* h_grid, int nh, int part, int nparts,
                         const float* d_ew_all, double* partial_logL, int64_t* evals) {
    if (!c || !p || !h_grid || nh <= 0 || !partial_logL || nparts <= 0 || part < 0 || part >= nparts)
        return mgk_fail(c, MGK_ERR_INVALID, "loo_share_loglik: bad arguments");
    float lo, hi;
    int st = check_bandwidths(c, h_grid, nh, &lo, &hi);
    if (st) return st;
    mgk_loo_batch* B = nullptr;
    if ((st = mgk_loo_batch_create_share(c, p, nullptr, lo, hi, nh, part, nparts, d_ew_all,
                                         share_chunk(p->n, nparts), &B, false)))  // runs once: no graph
        return st;
    st = mgk_loo_batch_run(B, h_grid, partial_logL, nullptr, nullptr, evals);
    mgk_loo_batch_destroy(B);
    return st;
}

int mgk_mle_fixed_bandwidth(mgk_ctx* c, mgk_points* p, const mgk_raster* r, float h0, float* h_opt, int* iterations) {
    if (!c || !p || !h_opt || !(h0 > 0.0f)) return mgk_fail(c, MGK_ERR_INVALID, "mle_fixed_bandwidth: bad arguments");
    if (r && !p->has_dist2) return mgk_fail(c, MGK_ERR_INVALID, "loo: run mgk_boundary_dist first");
    if (r && !cap_covers(p, 2 * h0))  // every probe lies in [h0/20, 2 h0]
        return mgk_fail(c, MGK_ERR_INVALID, "loo: the boundary distances are exact only within " +
                                                std::to_string(p->dist2_cap) + ", less than 3 h_max");
    // MLE_FixedBandWidth, kde_cuda_kdtr_tiled.cu:3044-3093 (float bracket arithmetic)
    float hA = h0 / 20;
    float hD = 2 * h0;
    float width = hD - hA;
    const float epsilon = width / 100;
    const float factor = 1 + sqrtf(5.0f);
    mgk_loo_batch* B = nullptr;
    int st = mgk_loo_batch_create(c, p, r, hA, hD, 2, &B);  // every probe lies in [h0/20, 2 h0]
    if (st) return st;
    int it = 0;
    while (width > epsilon && it < 30) {
        const float hB = hA + width / factor;
        const float hC = hD - width / factor;
        const float hh[2] = {hB, hC};
        double l[2];
        if ((st = mgk_loo_batch_run(B, hh, l, nullptr, nullptr, nullptr))) break;
        if (l[0] > l[1]) hD = hC;
        else hA = hB;
        width = hD - hA;
        it++;
    }
    mgk_loo_batch_destroy(B);
    if (st) return st;
    *h_opt = (hA + hD) / 2;
    if (iterations) *iterations = it;
    return MGK_OK;
}

// ---------------------------------------------------------- whole raster --
// The tiles go through a three-stream pipeline: the mask of tile k+1 is
// copied in (stream h2d) and the density of tile k-1 copied out (stream d2h)
// while tile k is computed on the context stream, with two device buffers
// of each kind and events between the stages.  Without an explicit tile
// side the raster is cut into full-width bands of about an eighth of its
// rows (at least 256, a multiple of the 64-row density block), so that the
// copies in and out hide under the density of the neighbouring bands.  The
// last 256 rows form a band of their own: its copy out follows the last
// density launch with nothing left to hide it, so it is kept short.
#ifndef MGK_RASTER_BANDS
#define MGK_RASTER_BANDS 8
#endif
// device buffers of each kind (mask in, density out) in flight
#ifndef MGK_RASTER_DEPTH
#define MGK_RASTER_DEPTH 3
#endif

namespace {
constexpr int64_t kRasterBands = MGK_RASTER_BANDS;  // full-width bands without an explicit tile side
constexpr int kDepth = MGK_RASTER_DEPTH;

// cuStreamWaitValue32 / cuStreamWriteValue32 through the runtime's driver
// entry points (no link-time dependency on the driver library).
struct StreamMemOps {
    PFN_cuStreamWaitValue32_v11070 wait = nullptr;
    PFN_cuStreamWriteValue32_v11070 write = nullptr;
};
const StreamMemOps& stream_memops() {
    static StreamMemOps ops;
    static std::once_flag once;
    std::call_once(once, [] {
        void *w = nullptr, *v = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        if (cudaGetDriverEntryPointByVersion("cuStreamWaitValue32", &w, 11070, cudaEnableDefault, &q1) ==
                cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPointByVersion("cuStreamWriteValue32", &v, 11070, cudaEnableDefault, &q2) ==
                cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess) {
            ops.wait = reinterpret_cast<PFN_cuStreamWaitValue32_v11070>(w);
            ops.write = reinterpret_cast<PFN_cuStreamWriteValue32_v11070>(v);
        }
        (void)cudaGetLastError();
    });
    return ops;
}

// Whether stream memory operations work on the context's device: checked
// once per device with a write and a wait that the write satisfies.
bool stream_memops_work(mgk_ctx* c) {
    static std::mutex mu;
    static std::map<int, bool> ok_by_device;
    std::lock_guard<std::mutex> lk(mu);
    auto f = ok_by_device.find(c->device);
    if (f != ok_by_device.end()) return f->second;
    const StreamMemOps& ops = stream_memops();
    bool ok = false;
    void* d = nullptr;
    if (ops.wait && ops.write && mgk_alloc(c, &d, 256) == MGK_OK) {
        const CUdeviceptr a = (CUdeviceptr)(uintptr_t)d;
        ok = ops.write((CUstream)c->stream, a, 1u, CU_STREAM_WRITE_VALUE_DEFAULT) == CUDA_SUCCESS &&
             ops.wait((CUstream)c->stream, a, 1u, CU_STREAM_WAIT_VALUE_GEQ) == CUDA_SUCCESS &&
             cudaStreamSynchronize(c->stream) == cudaSuccess;
        (void)cudaGetLastError();
        mgk_free(c, d, 256);
    }
    ok_by_device[c->device] = ok;
    return ok;
}
struct RasterPipe {
    cudaStream_t h2d = nullptr, d2h = nullptr, alt = nullptr, mrg = nullptr;
    cudaEvent_t mask_ready[kDepth] = {}, done[kDepth] = {}, out_free[kDepth] = {}, dens[kDepth] = {};
    ~RasterPipe() {
        for (int i = 0; i < kDepth; i++) {
            if (mask_ready[i]) cudaEventDestroy(mask_ready[i]);
            if (done[i]) cudaEventDestroy(done[i]);
            if (out_free[i]) cudaEventDestroy(out_free[i]);
            if (dens[i]) cudaEventDestroy(dens[i]);
        }
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
        if (alt) cudaStreamDestroy(alt);
        if (mrg) cudaStreamDestroy(mrg);
    }
    cudaError_t init() {
        cudaError_t e = cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&alt, cudaStreamNonBlocking);
        // the merges of split blocks at the highest priority: a band's merge
        // is scheduled ahead of the next band's pending CTAs
        int least = 0, greatest = 0;
        if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&mrg, cudaStreamNonBlocking, greatest);
        for (int i = 0; i < kDepth && e == cudaSuccess; i++) {
            e = cudaEventCreateWithFlags(&mask_ready[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&out_free[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&dens[i], cudaEventDisableTiming);
        }
        return e;
    }
};
}  // namespace

// The whole path over rows [row_lo, row_hi) of dg (dmask and out_density
// hold those rows only).  A strict row range keeps, on the device, only the
// points within 3 h_max of its rows (the densities of its cells need no
// others), and out_ew must then be NULL.
// ---- bit-packed density masks --------------------------------------------
// The whole-raster path sends its NoData mask to the device as 1 bit per cell
// (1 = valid) instead of 32: with the density coming back over the same link,
// the float mask's upload set the pace of the bands (about 36 GB/s each way).
// Worker threads pack the bands in order, ahead of their uploads.

// One mask row: bit c % 8 of byte c / 8 is (src[c] != nodata), as the float
// kernels compare (so a NaN NoData value marks every cell valid); the row's
// padding bytes up to `bytes` are zero.
__attribute__((target("avx2"))) static void pack_mask_row_avx2(const float* src, int64_t n, float nodata,
                                                              unsigned char* dst, int64_t bytes) {
    const __m256 nd = _mm256_set1_ps(nodata);
    int64_t c = 0;
    for (; c + 8 <= n; c += 8)
        dst[c >> 3] = (unsigned char)_mm256_movemask_ps(_mm256_cmp_ps(_mm256_loadu_ps(src + c), nd, _CMP_NEQ_UQ));
    int64_t b = c >> 3;
    if (c < n) {
        unsigned v = 0;
        for (int64_t k = c; k < n; k++) v |= (unsigned)(src[k] != nodata) << (k - c);
        dst[b++] = (unsigned char)v;
    }
    for (; b < bytes; b++) dst[b] = 0;
}

static void pack_mask_row(const float* src, int64_t n, float nodata, unsigned char* dst, int64_t bytes) {
    int64_t b = 0;
    for (int64_t c = 0; c < n; c += 8, b++) {
        unsigned v = 0;
        for (int64_t k = c; k < std::min<int64_t>(n, c + 8); k++) v |= (unsigned)(src[k] != nodata) << (k - c);
        dst[b] = (unsigned char)v;
    }
    for (; b < bytes; b++) dst[b] = 0;
}

#ifndef MGK_MASK_PACK_THREADS
#define MGK_MASK_PACK_THREADS 8  // at most this many, and at most half the host's hardware threads
#endif

class MaskPacker {
  public:
    // rows [band_r0[k] - row_lo, band_r0[k + 1] - row_lo) of src form band k
    MaskPacker(const float* src, int64_t ncols, float nodata, unsigned char* dst, int64_t stride,
               const std::vector<int64_t>& band_r0, int64_t row_lo)
        : src_(src), ncols_(ncols), nodata_(nodata), dst_(dst), stride_(stride),
          avx2_(__builtin_cpu_supports("avx2")) {
        const int64_t nb = (int64_t)band_r0.size() - 1;
        band_rows_.resize(nb);
        done_ = std::vector<std::atomic<int64_t>>(nb);
        for (int64_t k = 0; k < nb; k++) {
            band_rows_[k] = band_r0[k + 1] - band_r0[k];
            done_[k].store(0);
            for (int64_t r = band_r0[k]; r < band_r0[k + 1]; r += kChunk)
                chunks_.push_back({k, r - row_lo, std::min<int64_t>(band_r0[k + 1], r + kChunk) - r});
        }
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nt = (int)std::min<unsigned>(MGK_MASK_PACK_THREADS, std::max(1u, hw / 2));
        for (int t = 0; t < nt; t++) threads_.emplace_back([this] { work(); });
    }
    ~MaskPacker() {
        stop_.store(true);
        for (std::thread& t : threads_) t.join();
    }
    // returns once band k is packed
    void wait_band(int64_t k) {
        while (done_[k].load(std::memory_order_acquire) < band_rows_[k]) std::this_thread::yield();
    }

  private:
    struct Chunk {
        int64_t band, row, rows;
    };
    static constexpr int64_t kChunk = 64;
    void work() {
        for (;;) {
            const int64_t i = next_.fetch_add(1);
            if (i >= (int64_t)chunks_.size() || stop_.load()) return;
            const Chunk& ch = chunks_[i];
            for (int64_t r = ch.row; r < ch.row + ch.rows; r++) {
                if (avx2_) pack_mask_row_avx2(src_ + r * ncols_, ncols_, nodata_, dst_ + r * stride_, stride_);
                else pack_mask_row(src_ + r * ncols_, ncols_, nodata_, dst_ + r * stride_, stride_);
            }
            done_[ch.band].fetch_add(ch.rows, std::memory_order_release);
        }
    }
    const float* src_;
    int64_t ncols_;
    float nodata_;
    unsigned char* dst_;
    int64_t stride_;
    bool avx2_;
    std::vector<Chunk> chunks_;
    std::vector<int64_t> band_rows_;
    std::vector<std::atomic<int64_t>> done_;
    std::atomic<int64_t> next_{0};
    std::atomic<bool> stop_{false};
    std::vector<std::thread> threads_;
};

static int kde_raster_rows(mgk_ctx* c, int64_t n, const float* x, const float* y, const float* w, const float* h_pp,
                           float h, int edge_correction, const mgk_grid* eg, const float* emask, const mgk_grid* dg,
                           int64_t row_lo, int64_t row_hi, const float* dmask, int64_t tile_side,
                           float* out_density, float* out_ew, int64_t* evals) {
    if (!c || !grid_ok(dg) || !out_density || (edge_correction && (!grid_ok(eg) || !emask)) ||
        (!h_pp && !(h > 0.0f)) || row_lo < 0 || row_hi > dg->nrows || row_lo >= row_hi)
        return mgk_fail(c, MGK_ERR_INVALID, "kde_raster: bad arguments");
    const bool part_rows = row_lo > 0 || row_hi < dg->nrows;
    if (part_rows && out_ew) return mgk_fail(c, MGK_ERR_INVALID, "kde_raster_rows: out_ew needs the whole raster");
    const int64_t nrows = row_hi - row_lo;
    // tile grid (kde_cuda_kdtr_tiled.cu:1373-1517 walks tiles row-major)
    int64_t tr, tc;
    const int64_t T = tile_side > 0 ? tile_side : c->tile_side;
    std::vector<int64_t> band_r0;  // full-width bands: first row of band k, then row_hi
    if (T > 0) {
        tr = std::min<int64_t>(T, nrows);
        tc = std::min<int64_t>(T, dg->ncols);
    } else {
        tr = std::max<int64_t>(256, ((nrows + kRasterBands - 1) / kRasterBands + 63) / 64 * 64);
        tr = std::min<int64_t>(tr, nrows);
        tc = dg->ncols;
        // the last band: the rows from the first 64-row block boundary at
        // most 256 rows before the end (band boundaries are block boundaries,
        // and no band is taller than tr)
        const int64_t tail_r0 = nrows > 2 * 256 ? row_lo + (nrows - 256 + 63) / 64 * 64 : row_hi;
        for (int64_t r0 = row_lo; r0 < tail_r0; r0 += tr) band_r0.push_back(r0);
        if (tail_r0 < row_hi) band_r0.push_back(tail_r0);
        band_r0.push_back(row_hi);
    }
    const int64_t ntc = (dg->ncols + tc - 1) / tc;
    const int64_t ntiles = band_r0.empty() ? (nrows + tr - 1) / tr * ntc : (int64_t)band_r0.size() - 1;
    const size_t tb = sizeof(float) * (size_t)tr * (size_t)tc;
    // full-width bands take the mask as bits (rows of mstride bytes, a
    // multiple of 16); explicit tiles take it as floats
    const bool packed = dmask && !band_r0.empty();
    const int64_t mstride = (dg->ncols + 127) / 128 * 16;
    const size_t tbm = packed ? (size_t)tr * (size_t)mstride : tb;
    RasterPipe pipe;
    cudaError_t ce = pipe.init();
    if (ce != cudaSuccess) return mgk_cuda_fail(c, ce, "kde_raster streams");
    mgk_points* p = nullptr;
    mgk_raster* em = nullptr;
    mgk_index* idx = nullptr;
    float* d_mask[kDepth] = {};
    float* d_out[kDepth] = {};
    int64_t ev_edge = 0, ev_den = 0;
    const float hfix = h_pp ? 0.0f : h;
    int st = MGK_OK;
    for (int i = 0; i < (int)std::min<int64_t>(ntiles, kDepth) && st == MGK_OK; i++) {
        st = mgk_alloc(c, (void**)&d_out[i], tb);
        if (st == MGK_OK && dmask) st = mgk_alloc(c, (void**)&d_mask[i], tbm);
    }
    // the packed mask of all rows, in page-locked memory (staging slot 3),
    // filled band by band by the packer's threads while the GPU works
    unsigned char* h_bits = nullptr;
    std::unique_ptr<MaskPacker> packer;
    if (st == MGK_OK && packed) {
        void* dev_alias = nullptr;
        st = mgk_host_stage_slot(c, 3, (size_t)nrows * (size_t)mstride, (void**)&h_bits, &dev_alias);
        if (st == MGK_OK)
            packer.reset(new MaskPacker(dmask, dg->ncols, dg->nodata, h_bits, mstride, band_r0, row_lo));
    }
    auto tile_of = [&](int64_t k, int64_t& r0, int64_t& c0, int64_t& nr, int64_t& nc) {
        if (!band_r0.empty()) {
            r0 = band_r0[k];
            nr = std::min<int64_t>(band_r0[k + 1], r0 + tr) - r0;
            c0 = 0;
            nc = dg->ncols;
            return;
        }
        r0 = row_lo + (k / ntc) * tr;
        c0 = (k % ntc) * tc;
        nr = std::min<int64_t>(tr, row_hi - r0);
        nc = std::min<int64_t>(tc, dg->ncols - c0);
    };
    // mask of tile k into buffer k % kDepth, after the density of tile k - kDepth read it
    auto mask_in = [&](int64_t k) -> cudaError_t {
        if (!dmask || k >= ntiles) return cudaSuccess;
        int64_t r0, c0, nr, nc;
        tile_of(k, r0, c0, nr, nc);
        const int b = (int)(k % kDepth);
        cudaError_t e = k >= kDepth ? cudaStreamWaitEvent(pipe.h2d, pipe.done[b], 0) : cudaSuccess;
        if (e == cudaSuccess && packed) {
            packer->wait_band(k);
            e = cudaMemcpyAsync(d_mask[b], h_bits + (r0 - row_lo) * mstride, (size_t)nr * (size_t)mstride,
                                cudaMemcpyHostToDevice, pipe.h2d);
        } else if (e == cudaSuccess) {
            e = cudaMemcpy2DAsync(d_mask[b], sizeof(float) * nc, dmask + (r0 - row_lo) * dg->ncols + c0,
                                  sizeof(float) * dg->ncols, sizeof(float) * nc, nr, cudaMemcpyHostToDevice, pipe.h2d);
        }
        if (e == cudaSuccess) e = cudaEventRecord(pipe.mask_ready[b], pipe.h2d);
        return e;
    };
    // the density kernels' eval counter and staging-wait flag (counters 4 and
    // 7, shared by all tiles), zeroed before any copy is in flight
    if (st == MGK_OK && (ce = cudaMemsetAsync(c->d_counter + 4, 0, 4 * sizeof(unsigned long long), c->stream)) !=
                            cudaSuccess)
        st = mgk_cuda_fail(c, ce, "kde_raster counters");
    if (st == MGK_OK) st = mgk_points_upload(c, n, x, y, w, h_pp, &p);
    if (st == MGK_OK && part_rows) {
        // the halo of the rows: points within 3 h_max of their cell centres
        float hmax = h;
        if (h_pp)
            for (int64_t i = 0; i < n; i++) hmax = std::max(hmax, h_pp[i]);
        const double reach = 3.0 * (double)hmax * (1.0 + 1e-6) + 1e-6 * (double)dg->cs;
        const double y_top = (double)mgk_cell_y(dg->yll, dg->cs, dg->nrows, row_lo);
        const double y_bot = (double)mgk_cell_y(dg->yll, dg->cs, dg->nrows, row_hi - 1);
        mgk_points* q = nullptr;
        st = mgk_points_select(c, p, -DBL_MAX, DBL_MAX, y_bot - reach, y_top + reach, &q);
        mgk_points_destroy(p);
        p = q;
    }
    // The edge mask travels on the copy stream while the index is built from
    // the points (its records take the edge weights once they are known).
    float* d_em = nullptr;
    const size_t b_em = edge_correction ? sizeof(float) * (size_t)eg->ncols * (size_t)eg->nrows : 0;
    cudaEvent_t em_ready = nullptr;
    if (st == MGK_OK && edge_correction) {
        if ((st = mgk_alloc(c, (void**)&d_em, b_em)) == MGK_OK) {
            ce = cudaEventCreateWithFlags(&em_ready, cudaEventDisableTiming);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_em, emask, b_em, cudaMemcpyHostToDevice, pipe.h2d);
            if (ce == cudaSuccess) ce = cudaEventRecord(em_ready, pipe.h2d);
            if (ce != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster edge mask");
        }
        if (st == MGK_OK) st = mgk_raster_wrap(c, eg, d_em, &em);
    }
    // the first tile's float mask travels while the points are prepared (a
    // packed band's bits follow the counts: the packer may still be at work)
    if (st == MGK_OK && !packed && (ce = mask_in(0)) != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster mask");
    if (st == MGK_OK) st = mgk_index_build(c, p, hfix, 0.0f, &idx);
    if (st == MGK_OK) {
        if (edge_correction) {
            // distances exact up to 3 h_max: all the edge-weight short-circuit reads
            float hmax = h;
            if (h_pp)
                for (int64_t i = 0; i < n; i++) hmax = std::max(hmax, h_pp[i]);
            const double reach = 3.0 * (double)hmax * (1.0 + 1e-6);
            if ((ce = cudaStreamWaitEvent(c->stream, em_ready, 0)) != cudaSuccess)
                st = mgk_cuda_fail(c, ce, "kde_raster edge mask");
            if (st == MGK_OK && (st = mgk_boundary_dist_within(c, p, em, reach)) == MGK_OK &&
                (st = mgk_edge_weights(c, p, em, hfix, evals ? &ev_edge : nullptr)) == MGK_OK)
                st = mgk_index_refresh_weights(c, idx, p);
        } else {
            st = mgk_edge_weights_unit(c, p);  // w * 1: the records built above hold the same weights
        }
    }
    if (st == MGK_OK && out_ew) {
        ce = cudaMemcpyAsync(out_ew, p->ew, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream);
        if (ce != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster ew");
    }
    // density of tile k out, after its kernels (event done) and into the host raster
    auto out_copy = [&](int64_t k) -> cudaError_t {
        if (k < 0) return cudaSuccess;
        int64_t r0, c0, nr, nc;
        tile_of(k, r0, c0, nr, nc);
        const int b = (int)(k % kDepth);
        cudaError_t e = cudaStreamWaitEvent(pipe.d2h, pipe.done[b], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(out_density + (r0 - row_lo) * dg->ncols + c0, sizeof(float) * dg->ncols, d_out[b],
                                  sizeof(float) * nc, sizeof(float) * nc, nr, cudaMemcpyDeviceToHost, pipe.d2h);
        if (e == cudaSuccess) e = cudaEventRecord(pipe.out_free[b], pipe.d2h);
        return e;
    };
    // Tile k's plan is made while tile k - 1 computes: the counting kernel of
    // tile k is queued ahead of tile k - 1's density on the same stream, so
    // the host can plan from its counts (staging slot 1 + k % 2) while that
    // density runs, and the next density launch follows without a gap.  When
    // the counting kernel of tile k has finished, the density of tile k - 2
    // (queued before it) has too, so that plan and its staging slot are free.
    mgk_dplan* plans[2] = {nullptr, nullptr};
    cudaEvent_t counted = nullptr;
    if (st == MGK_OK && (ce = cudaEventCreateWithFlags(&counted, cudaEventDisableTiming)) != cudaSuccess)
        st = mgk_cuda_fail(c, ce, "kde_raster event");
    unsigned long long* d_ev = evals ? c->d_counter + 4 : nullptr;
    auto plan_of = [&](int64_t k) -> int {  // after tile k's counting kernel has finished
        int64_t r0, c0, nr, nc;
        tile_of(k, r0, c0, nr, nc);
        const int b = (int)(k & 1), db = (int)(k % kDepth);
        mgk_density_discard(c, plans[b]);  // tile k - 2's
        plans[b] = nullptr;
        return mgk_density_plan_counted(c, idx, dg, r0, c0, nr, nc, d_mask[db], d_out[db], d_ev, 1 + b, &plans[b]);
    };
    auto count_of = [&](int64_t k) -> int {
        int64_t r0, c0, nr, nc;
        tile_of(k, r0, c0, nr, nc);
        return mgk_density_counts_launch(c, idx, dg, r0, c0, nr, nc, 1 + (int)(k & 1), c->stream);
    };
    // both slots sized up front for a full tile's counts and work list, so a
    // counting launch never has to regrow a slot whose previous plan may still
    // be running
    for (int i = 1; i <= 2 && st == MGK_OK; i++) {
        void *hs = nullptr, *ds = nullptr;
        const size_t nblk = (size_t)((tr + 63) / 64) * (size_t)((tc + 127) / 128);
        st = mgk_host_stage_slot(c, i, 64 * nblk + 4096, &hs, &ds);
    }
    std::vector<mgk_dplan*> band_plans;
    unsigned* d_flag = nullptr;  // [band] its last CTA has started
    if (st == MGK_OK && !band_r0.empty()) {
        // ---- full-width bands ----
        // One count of all rows; each band planned from its slice while the
        // one before computes.  With stream memory operations the bands
        // alternate over two streams and band k waits for band k - 1's last
        // CTA to start, so its CTAs fill the SMs that band k - 1's tail
        // frees; a stream write after each band ends that wait in any case.
        // MGK_RASTER_ONE_STREAM=1 forces the one-stream schedule, the one
        // taken without stream memory operations (same plans, same raster)
        const StreamMemOps& ops = stream_memops();
        const char* one = std::getenv("MGK_RASTER_ONE_STREAM");
        const bool two = !(one && one[0] == '1') && stream_memops_work(c);
        if (two && (st = mgk_alloc(c, (void**)&d_flag, sizeof(unsigned) * ntiles)) == MGK_OK &&
            (ce = cudaMemsetAsync(d_flag, 0, sizeof(unsigned) * ntiles, c->stream)) != cudaSuccess)
            st = mgk_cuda_fail(c, ce, "kde_raster flags");
        if (st == MGK_OK) st = mgk_density_counts_launch(c, idx, dg, row_lo, 0, nrows, dg->ncols, 0, c->stream);
        if (st == MGK_OK && packed && (ce = mask_in(0)) != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster mask");
        if (st == MGK_OK && (ce = cudaStreamSynchronize(c->stream)) != cudaSuccess)
            st = mgk_cuda_fail(c, ce, "kde_raster plan");
        // the alternate stream follows the preparation on the context stream
        if (st == MGK_OK && two && ((ce = cudaEventRecord(counted, c->stream)) != cudaSuccess ||
                                    (ce = cudaStreamWaitEvent(pipe.alt, counted, 0)) != cudaSuccess))
            st = mgk_cuda_fail(c, ce, "kde_raster");
        const int64_t* counts = st == MGK_OK ? mgk_density_counts_host(c, 0) : nullptr;
        const int64_t nbx = (dg->ncols + 127) / 128;
        band_plans.assign(ntiles, nullptr);
        for (int64_t k = 1; k < kDepth - 1 && st == MGK_OK; k++)
            if ((ce = mask_in(k)) != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster mask");
        for (int64_t k = 0; st == MGK_OK && k < ntiles; k++) {
            const int db = (int)(k % kDepth);
            const cudaStream_t ks = two && (k & 1) ? pipe.alt : c->stream;
            // band k - 2 staged its work list from the same slot before its density
            if (k >= 2 && (ce = cudaEventSynchronize(pipe.done[(k - 2) % kDepth])) != cudaSuccess) {
                st = mgk_cuda_fail(c, ce, "kde_raster plan");
                break;
            }
            const int64_t r0 = band_r0[k], nr = band_r0[k + 1] - r0;
            if (nr > tr || (r0 - row_lo) % 64) {  // the buffers hold tr rows; plans slice whole block rows
                st = mgk_fail(c, MGK_ERR_INVALID, "kde_raster: band layout");
                break;
            }
            if ((st = mgk_density_plan_from_counts(c, idx, dg, r0, 0, nr, dg->ncols, counts + (r0 - row_lo) / 64 * nbx,
                                                   packed ? nullptr : d_mask[db], d_out[db], d_ev, 1 + (int)(k & 1),
                                                   &band_plans[k])))
                break;
            if (packed)
                mgk_density_set_mask_bits(band_plans[k], reinterpret_cast<const unsigned char*>(d_mask[db]), mstride);
            if (two) mgk_density_set_tail_flag(band_plans[k], d_flag + k);
            ce = dmask ? cudaStreamWaitEvent(ks, pipe.mask_ready[db], 0) : cudaSuccess;
            if (ce == cudaSuccess && k >= kDepth) ce = cudaStreamWaitEvent(ks, pipe.out_free[db], 0);
            if (ce != cudaSuccess) {
                st = mgk_cuda_fail(c, ce, "kde_raster tile");
                break;
            }
            if (two && k >= 1 &&
                ops.wait((CUstream)ks, (CUdeviceptr)(uintptr_t)(d_flag + k - 1), 1u, CU_STREAM_WAIT_VALUE_GEQ) != CUDA_SUCCESS) {
                st = mgk_fail(c, MGK_ERR_CUDA, "kde_raster: stream wait failed");
                break;
            }
            bool merged_on_mrg = false;
            if ((st = mgk_density_launch_split(c, band_plans[k], ks, pipe.mrg, pipe.dens[db], &merged_on_mrg))) break;
            if (two && ops.write((CUstream)ks, (CUdeviceptr)(uintptr_t)(d_flag + k), 1u, CU_STREAM_WRITE_VALUE_DEFAULT) !=
                           CUDA_SUCCESS) {
                st = mgk_fail(c, MGK_ERR_CUDA, "kde_raster: stream write failed");
                break;
            }
            ce = cudaEventRecord(pipe.done[db], merged_on_mrg ? pipe.mrg : ks);
            if (ce == cudaSuccess) ce = out_copy(k);
            // the mask of band k + kDepth - 1 (into the buffer band k - 1 read),
            // after band k is queued: a packed band may still be at the packer
            if (ce == cudaSuccess) ce = mask_in(k + kDepth - 1);
            if (ce != cudaSuccess) {
                st = mgk_cuda_fail(c, ce, "kde_raster tile");
                break;
            }
        }
    }
    if (st == MGK_OK && band_r0.empty() && ntiles > 0 && (st = count_of(0)) == MGK_OK) {
        if ((ce = cudaStreamSynchronize(c->stream)) != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster plan");
        else st = plan_of(0);
    }
    // the masks of the first kDepth - 1 tiles are on their way; tile k's loop
    // step sends the one of tile k + kDepth - 1 (its buffer's last reader is
    // tile k - 1's density)
    for (int64_t k = 1; k < kDepth - 1 && st == MGK_OK && band_r0.empty(); k++)
        if ((ce = mask_in(k)) != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster mask");
    for (int64_t k = 0; st == MGK_OK && band_r0.empty() && k < ntiles; k++) {
        const int b = (int)(k & 1), db = (int)(k % kDepth);
        ce = mask_in(k + kDepth - 1);
        if (ce != cudaSuccess) {
            st = mgk_cuda_fail(c, ce, "kde_raster mask");
            break;
        }
        if (k + 1 < ntiles) {
            if ((st = count_of(k + 1))) break;
            if ((ce = cudaEventRecord(counted, c->stream)) != cudaSuccess) {
                st = mgk_cuda_fail(c, ce, "kde_raster");
                break;
            }
        }
        const cudaStream_t ks = c->stream;
        if (dmask) ce = cudaStreamWaitEvent(ks, pipe.mask_ready[db], 0);
        if (ce == cudaSuccess && k >= kDepth) ce = cudaStreamWaitEvent(ks, pipe.out_free[db], 0);
        if (ce != cudaSuccess) {
            st = mgk_cuda_fail(c, ce, "kde_raster tile");
            break;
        }
        if ((st = mgk_density_launch_plan(c, plans[b], ks))) break;
        ce = cudaEventRecord(pipe.done[db], ks);
        if (ce == cudaSuccess) ce = out_copy(k);
        if (ce != cudaSuccess) {
            st = mgk_cuda_fail(c, ce, "kde_raster tile");
            break;
        }
        if (k + 1 < ntiles) {
            if ((ce = cudaEventSynchronize(counted)) != cudaSuccess) {
                st = mgk_cuda_fail(c, ce, "kde_raster plan");
                break;
            }
            st = plan_of(k + 1);
        }
    }
    // every copy and kernel of this call ends before its buffers are released
    if ((ce = cudaStreamSynchronize(pipe.h2d)) != cudaSuccess && st == MGK_OK) st = mgk_cuda_fail(c, ce, "kde_raster");
    if ((ce = cudaStreamSynchronize(pipe.d2h)) != cudaSuccess && st == MGK_OK) st = mgk_cuda_fail(c, ce, "kde_raster");
    if ((ce = cudaStreamSynchronize(c->stream)) != cudaSuccess && st == MGK_OK) st = mgk_cuda_fail(c, ce, "kde_raster");
    if ((ce = cudaStreamSynchronize(pipe.alt)) != cudaSuccess && st == MGK_OK) st = mgk_cuda_fail(c, ce, "kde_raster");
    if ((ce = cudaStreamSynchronize(pipe.mrg)) != cudaSuccess && st == MGK_OK) st = mgk_cuda_fail(c, ce, "kde_raster");
    for (int i = 0; i < 2; i++) mgk_density_discard(c, plans[i]);  // every kernel has ended
    for (mgk_dplan* D : band_plans) mgk_density_discard(c, D);
    if (d_flag) mgk_free(c, d_flag, sizeof(unsigned) * ntiles);
    if (counted) cudaEventDestroy(counted);
    if (st == MGK_OK) {  // counters 4 (density evals) and 7 (staging-wait flag)
        ce = cudaMemcpy(c->h_counter + 4, c->d_counter + 4, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) st = mgk_cuda_fail(c, ce, "kde_raster counters");
        else if (c->h_counter[7]) st = mgk_fail(c, MGK_ERR_TIMEOUT, "density: a shared-memory staging wait timed out");
        else ev_den = (int64_t)c->h_counter[4];
    }
    for (int i = 0; i < kDepth; i++) {
        if (d_out[i]) mgk_free(c, d_out[i], tb);
        if (d_mask[i]) mgk_free(c, d_mask[i], tbm);
    }
    mgk_index_destroy(idx);
    mgk_raster_destroy(em);
    if (d_em) mgk_free(c, d_em, b_em);
    if (em_ready) cudaEventDestroy(em_ready);
    mgk_points_destroy(p);
    if (st == MGK_OK && evals) *evals = ev_den + ev_edge;
    return st;
}

int mgk_kde_raster(mgk_ctx* c, int64_t n, const float* x, const float* y, const float* w, const float* h_pp, float h,
                   int edge_correction, const mgk_grid* eg, const float* emask, const mgk_grid* dg,
                   const float* dmask, int64_t tile_side, float* out_density, float* out_ew, int64_t* evals) {
    if (!dg) return mgk_fail(c, MGK_ERR_INVALID, "kde_raster: bad arguments");
    return kde_raster_rows(c, n, x, y, w, h_pp, h, edge_correction, eg, emask, dg, 0, dg->nrows, dmask, tile_side,
                           out_density, out_ew, evals);
}

int mgk_kde_raster_rows(mgk_ctx* c, int64_t n, const float* x, const float* y, const float* w, const float* h_pp,
                        float h, int edge_correction, const mgk_grid* eg, const float* emask, const mgk_grid* dg,
                        int64_t row0, int64_t nrows, const float* dmask_rows, int64_t tile_side, float* out_rows,
                        int64_t* evals) {
    if (!dg) return mgk_fail(c, MGK_ERR_INVALID, "kde_raster_rows: bad arguments");
    return kde_raster_rows(c, n, x, y, w, h_pp, h, edge_correction, eg, emask, dg, row0, row0 + nrows, dmask_rows,
                           tile_side, out_rows, nullptr, evals);
}

}  // extern "C"
