// Serving loop: KDE requests of uneven size with continuous batching.
//
// The reference has no server: it runs one study per process invocation
// (main, kde_cuda_kdtr_tiled.cu:290-1540).  Here a worker thread owns one
// context (one stream, one device allocator under an HBM budget) and serves a
// queue of requests, each a whole fixed-bandwidth KDE (points, bandwidth,
// density raster and optional mask, optional edge correction):
//
//  * admission: a queued request becomes active when the number of active
//    requests is below the slot count and its estimated device footprint fits
//    beside the active ones inside the budget; among the queued requests the
//    one with the most tiles goes first (largest first keeps a big request
//    from running alone at the end of a burst);
//  * preparation: its points, index (and edge-correction weights) are built
//    and stay resident on the device while it is active.  A second thread
//    with a context of its own does this (admission, preparation, and the
//    release of finished requests' memory), so new requests are prepared on
//    the GPU while the worker's ticks run;
//  * ticks: each tick takes the next tiles of every active request (row-major
//    tiles of tile_side x tile_side cells; one each when kTickTiles or more
//    requests are active, else up to kTickTiles / active each, so that a
//    request running alone still fills the GPU) and runs all of them in one
//    density launch (mgk_launch_density_jobs).  Each request has
//    2 kTickTiles device output tiles: a tick's results are copied to the
//    requests' host outputs on a second stream while the next tick computes
//    into the other tiles.
//    Requests admitted between ticks join the next tick, so a short request
//    that arrives while a large one is running finishes after a few ticks
//    instead of waiting for the large one.  A request is complete when the
//    copy of its last tile has landed.
//
// Each tile is planned on its own, so a request's raster is bitwise the same
// whether it ran alone or in a mix.  Callers submit from any thread and wait
// or poll on a ticket; the host buffers of a request must stay valid until it
// completes.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "mgk_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

// Tiles a tick takes in all: one per active request when that many are
// active, else up to kTickTiles / active from each.
constexpr int kTickTiles = 4;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

__global__ void k_copy_counts(int n, const unsigned long long* __restrict__ src, volatile unsigned long long* dst) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// A kernel rather than a memset, so nothing on the context stream goes
// through a copy engine during a tick.
__global__ void k_zero_counts(int n, unsigned long long* __restrict__ a) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = 0ull;
}

struct Job {
    uint64_t id = 0;
    mgk_request req{};
    int state = 0;  // 0 queued, 1 active, 2 done
    int status = MGK_OK;
    uint64_t est = 0;
    Clock::time_point t_submit, t_start, t_done;
    mgk_points* p = nullptr;
    mgk_raster* em = nullptr;
    mgk_index* idx = nullptr;
    float* d_mask[kTickTiles] = {};  // the masks of a tick's tiles
    float* d_out[2 * kTickTiles] = {};  // tile k computes into d_out[k % (2 kTickTiles)]
    cudaEvent_t out_free[2 * kTickTiles] = {};  // the copy out of d_out[b] has finished
    bool used[2 * kTickTiles] = {};
    size_t tile_bytes = 0;
    int64_t tiles_x = 0, tiles_y = 0, next_tile = 0;
    int64_t evals = 0;
};

}  // namespace

namespace {
// The device resources of a request, handed to the preparation thread (whose
// context allocated them) for release once the request has finished.
struct Res {
    mgk_points* p = nullptr;
    mgk_raster* em = nullptr;
    mgk_index* idx = nullptr;
    float* d_mask[kTickTiles] = {};
    float* d_out[2 * kTickTiles] = {};
    cudaEvent_t out_free[2 * kTickTiles] = {};
    size_t tile_bytes = 0;
};
}  // namespace

struct mgk_server {
    mgk_ctx* ctx = nullptr;   // the worker's: ticks and copies
    mgk_ctx* pctx = nullptr;  // the preparation thread's: requests' points, indexes and tiles
    int64_t tile = 2048;
    int max_active = 8;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_prep;
    std::deque<Job*> queue;
    std::map<uint64_t, Job*> jobs;  // every job until its result is collected
    int preparing = 0;           // admitted, being prepared
    std::vector<Job*> active;    // tiles left to compute
    std::vector<Job*> draining;  // every tile computed, the last copies in flight
    std::vector<Res> to_release;
    std::thread prep;
    cudaStream_t d2h = nullptr;  // copies of finished tiles to the host
    unsigned long long* h_ev = nullptr;  // per-tick eval counts, mapped page-locked
    unsigned long long* d_ev_map = nullptr;  // their device address
    int ev_cap = 0;
    uint64_t reserved = 0;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    // statistics
    uint64_t ticks = 0, tiles = 0, max_batch = 0, completed = 0;
};

namespace {

// Device bytes a request holds while active (an upper estimate).
uint64_t estimate_bytes(const mgk_request& r, int64_t tile) {
    const uint64_t n = (uint64_t)std::max<int64_t>(r.n, 1);
    uint64_t b = n * 24;         // x, y, w, dist2, ew
    b += n * 64;                 // index records, permutation and sort scratch
    const double ext = std::max(r.grid.ncols, r.grid.nrows) * (double)r.grid.cs + 6.0 * r.h;
    const double side = std::max(0.5 * (double)r.h, ext / 4096.0);  // the default bin factor
    const double bins = std::min(4096.0 * 4096.0, std::pow(ext / side + 2.0, 2.0));
    b += (uint64_t)(bins * 4.0);
    if (r.edge) b += (uint64_t)r.edge_grid.ncols * (uint64_t)r.edge_grid.nrows * 24;
    const uint64_t tr = (uint64_t)std::min<int64_t>(tile, r.grid.nrows), tc = (uint64_t)std::min<int64_t>(tile, r.grid.ncols);
    b += 3 * kTickTiles * tr * tc * 4;                    // masks and output tiles
    b += ((tr + 63) / 64) * ((tc + 63) / 64) * 64 * 1024;  // split-block scratch and work list
    return b + b / 4 + (16u << 20);
}

// Density tiles of a request.
int64_t tile_count(const mgk_server* S, const mgk_request& r) {
    const int64_t tr = std::min<int64_t>(S->tile, r.grid.nrows), tc = std::min<int64_t>(S->tile, r.grid.ncols);
    return ((r.grid.nrows + tr - 1) / tr) * ((r.grid.ncols + tc - 1) / tc);
}

void release(mgk_ctx* pc, Res& R) {
    mgk_index_destroy(R.idx);
    mgk_raster_destroy(R.em);
    mgk_points_destroy(R.p);
    for (int b = 0; b < kTickTiles; b++) mgk_free(pc, R.d_mask[b], R.tile_bytes);
    for (int b = 0; b < 2 * kTickTiles; b++) {
        mgk_free(pc, R.d_out[b], R.tile_bytes);
        if (R.out_free[b]) cudaEventDestroy(R.out_free[b]);
    }
    R = Res{};
}

// Moves a request's device resources out of the job.
Res take(Job* J) {
    Res R;
    R.p = J->p;
    R.em = J->em;
    R.idx = J->idx;
    R.tile_bytes = J->tile_bytes;
    for (int b = 0; b < kTickTiles; b++) {
        R.d_mask[b] = J->d_mask[b];
        J->d_mask[b] = nullptr;
    }
    for (int b = 0; b < 2 * kTickTiles; b++) {
        R.d_out[b] = J->d_out[b];
        R.out_free[b] = J->out_free[b];
        J->d_out[b] = nullptr;
        J->out_free[b] = nullptr;
    }
    J->p = nullptr;
    J->em = nullptr;
    J->idx = nullptr;
    return R;
}

// Uploads and indexes a newly admitted request (preparation thread, its own
// context and stream); returns once the device holds all of it.
int prepare(mgk_server* S, Job* J) {
    mgk_ctx* c = S->pctx;
    const mgk_request& r = J->req;
    int st = mgk_points_upload(c, r.n, r.x, r.y, r.w, nullptr, &J->p);
    if (st) return st;
    if (r.edge) {
        int64_t ev = 0;
        if ((st = mgk_raster_upload(c, &r.edge_grid, r.edge_mask, &J->em))) return st;
        // distances exact up to 3h: all the edge-weight short-circuit reads
        if ((st = mgk_boundary_dist_within(c, J->p, J->em, 3.0 * (double)r.h * (1.0 + 1e-6)))) return st;
        if ((st = mgk_edge_weights(c, J->p, J->em, r.h, &ev))) return st;
        J->evals += ev;
    } else if ((st = mgk_edge_weights_unit(c, J->p))) {
        return st;
    }
    if ((st = mgk_index_build(c, J->p, r.h, 0.0f, &J->idx))) return st;
    const int64_t tr = std::min<int64_t>(S->tile, r.grid.nrows), tc = std::min<int64_t>(S->tile, r.grid.ncols);
    J->tile_bytes = sizeof(float) * (size_t)tr * (size_t)tc;
    J->tiles_x = (r.grid.ncols + tc - 1) / tc;
    J->tiles_y = (r.grid.nrows + tr - 1) / tr;
    const int64_t ntiles = J->tiles_x * J->tiles_y;
    const int nbuf = (int)std::min<int64_t>(ntiles, 2 * kTickTiles);
    for (int b = 0; b < nbuf; b++) {
        if ((st = mgk_alloc(c, (void**)&J->d_out[b], J->tile_bytes))) return st;
        const cudaError_t e = cudaEventCreateWithFlags(&J->out_free[b], cudaEventDisableTiming);
        if (e != cudaSuccess) return mgk_cuda_fail(c, e, "serve: event");
    }
    for (int b = 0; r.mask && b < (int)std::min<int64_t>(ntiles, kTickTiles); b++)
        if ((st = mgk_alloc(c, (void**)&J->d_mask[b], J->tile_bytes))) return st;
    J->next_tile = 0;
    const cudaError_t e = cudaStreamSynchronize(c->stream);  // the worker's stream reads all of it
    if (e != cudaSuccess) return mgk_cuda_fail(c, e, "serve: preparation");
    return MGK_OK;
}

// A request is done: its device memory goes to the preparation thread for
// release, and its waiters are told.
void finish(mgk_server* S, Job* J, int status) {
    Res R = take(J);
    std::lock_guard<std::mutex> lk(S->mu);
    S->to_release.push_back(R);
    S->cv_prep.notify_one();
    J->status = status;
    J->state = 2;
    J->t_done = Clock::now();
    S->reserved -= J->est;
    S->active.erase(std::remove(S->active.begin(), S->active.end(), J), S->active.end());
    S->draining.erase(std::remove(S->draining.begin(), S->draining.end(), J), S->draining.end());
    S->completed++;
    S->cv_done.notify_all();
}

// The copy out of a job's last tile: its buffer's out_free event.
cudaEvent_t last_copy(const Job* J) { return J->out_free[(J->next_tile - 1) % (2 * kTickTiles)]; }

// Completes the draining jobs whose last copy has landed (all of them when
// wait is set).
void reap(mgk_server* S, bool wait) {
    std::vector<Job*> d;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        d = S->draining;
    }
    for (Job* J : d) {
        cudaError_t e = wait ? cudaEventSynchronize(last_copy(J)) : cudaEventQuery(last_copy(J));
        if (e == cudaErrorNotReady) {
            (void)cudaGetLastError();
            continue;
        }
        finish(S, J, e == cudaSuccess ? MGK_OK : mgk_cuda_fail(S->ctx, e, "serve: tile copy"));
    }
}

// One tick: the next tiles of every active, prepared request in one launch
// (up to kTickTiles / active each, at least one); the tiles' copies to the
// host are queued on the copy stream and overlap the next tick.
void tick(mgk_server* S, std::vector<Job*>& act) {
    mgk_ctx* c = S->ctx;
    cudaStream_t s = c->stream;
    std::vector<mgk_tile_job> tj;
    std::vector<Job*> owner;
    std::vector<int64_t> r0s, c0s, tiles;
    const int quota = std::max(1, kTickTiles / std::max(1, (int)act.size()));
    int st = MGK_OK;
    for (Job* J : act) {
        const mgk_request& r = J->req;
        const int64_t tr = std::min<int64_t>(S->tile, r.grid.nrows), tc = std::min<int64_t>(S->tile, r.grid.ncols);
        const int64_t ntiles = J->tiles_x * J->tiles_y;
        for (int q = 0; q < quota && J->next_tile + q < ntiles && st == MGK_OK; q++) {
            const int64_t t = J->next_tile + q;
            const int64_t ty = t / J->tiles_x, tx = t % J->tiles_x;
            const int64_t r0 = ty * tr, c0 = tx * tc;
            const int64_t nr = std::min(tr, r.grid.nrows - r0), nc = std::min(tc, r.grid.ncols - c0);
            const int b = (int)(t % (2 * kTickTiles));
            // the tile buffer's previous copy out must have finished before it is rewritten
            if (J->used[b] && cudaStreamWaitEvent(s, J->out_free[b], 0) != cudaSuccess) {
                st = MGK_ERR_CUDA;
                break;
            }
            // a tick's masks: the previous tick's kernels read these buffers earlier on this stream
            if (r.mask) {
                const cudaError_t e = cudaMemcpy2DAsync(J->d_mask[q], sizeof(float) * nc, r.mask + r0 * r.grid.ncols + c0,
                                                        sizeof(float) * r.grid.ncols, sizeof(float) * nc, nr,
                                                        cudaMemcpyHostToDevice, s);
                if (e != cudaSuccess) {
                    st = mgk_cuda_fail(c, e, "serve: tile mask");
                    break;
                }
            }
            tj.push_back(mgk_tile_job{J->idx, r.grid, r0, c0, nr, nc, r.mask ? J->d_mask[q] : nullptr, J->d_out[b]});
            owner.push_back(J);
            r0s.push_back(r0);
            c0s.push_back(c0);
            tiles.push_back(t);
        }
        if (st) break;
    }
    unsigned long long* d_ev = nullptr;
    const size_t bev = sizeof(unsigned long long) * std::max<size_t>(tj.size(), 1);
    if (st == MGK_OK) st = mgk_alloc(c, (void**)&d_ev, bev);
    if (st == MGK_OK) {
        k_zero_counts<<<1, 256, 0, s>>>((int)std::max<size_t>(tj.size(), 1), d_ev);
        MGK_COUNT_LAUNCH(c, 1);
        if (cudaGetLastError() != cudaSuccess) st = MGK_ERR_CUDA;
    }
    if (st == MGK_OK && (int)tj.size() > S->ev_cap) st = mgk_fail(c, MGK_ERR_INVALID, "serve: more tiles than slots");
    if (st == MGK_OK) st = mgk_launch_density_jobs(c, (int)tj.size(), tj.data(), d_ev);  // returns after the kernels
    if (st == MGK_OK) {
        // eval counts into mapped host memory by a kernel: no copy engine, so
        // they do not wait behind the previous tick's tile copies
        k_copy_counts<<<1, 256, 0, s>>>((int)tj.size(), d_ev, S->d_ev_map);
        MGK_COUNT_LAUNCH(c, 1);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) st = MGK_ERR_CUDA;
    }
    mgk_free(c, d_ev, bev);
    std::vector<unsigned long long> ev(tj.size(), 0);
    if (st == MGK_OK)
        for (size_t k = 0; k < tj.size(); k++) ev[k] = S->h_ev[k];
    // copies of this tick's tiles to the host outputs, on the copy stream
    for (size_t k = 0; k < tj.size() && st == MGK_OK; k++) {
        Job* J = owner[k];
        const mgk_request& r = J->req;
        const int b = (int)(tiles[k] % (2 * kTickTiles));
        cudaError_t e = cudaMemcpy2DAsync(r.out + r0s[k] * r.grid.ncols + c0s[k], sizeof(float) * r.grid.ncols,
                                          tj[k].d_out, sizeof(float) * tj[k].ncols, sizeof(float) * tj[k].ncols,
                                          tj[k].nrows, cudaMemcpyDeviceToHost, S->d2h);
        if (e == cudaSuccess) e = cudaEventRecord(J->out_free[b], S->d2h);
        if (e != cudaSuccess) st = mgk_cuda_fail(c, e, "serve: tile result");
        J->used[b] = true;
    }
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->ticks++;
        S->tiles += tj.size();
        S->max_batch = std::max<uint64_t>(S->max_batch, tj.size());
    }
    for (Job* J : act) {
        if (st) {
            cudaStreamSynchronize(S->d2h);  // nothing of the job stays in flight
            finish(S, J, st);
            continue;
        }
        for (size_t k = 0; k < owner.size(); k++)
            if (owner[k] == J) {
                J->evals += (int64_t)ev[k];
                J->next_tile++;
            }
        if (J->next_tile == J->tiles_x * J->tiles_y) {
            std::lock_guard<std::mutex> lk(S->mu);
            S->active.erase(std::remove(S->active.begin(), S->active.end(), J), S->active.end());
            S->draining.push_back(J);
        }
    }
}

// The worker: ticks over the prepared requests and completes those whose
// last copy has landed.
void worker_main(mgk_server* S) {
    cudaSetDevice(S->ctx->device);
    for (;;) {
        reap(S, false);
        std::vector<Job*> act;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->active.empty()) {
                if (!S->draining.empty()) {
                    lk.unlock();
                    reap(S, true);  // nothing to compute: wait for the last copies
                    continue;
                }
                if (S->stop && S->queue.empty() && S->preparing == 0) return;
                S->cv_work.wait_for(lk, std::chrono::milliseconds(50));
                continue;
            }
            act = S->active;
        }
        tick(S, act);
    }
}

// The preparation thread: releases finished requests' memory, admits queued
// requests by free slots and the HBM budget (a request that fits nowhere
// alone is admitted when nothing else is in the server), prepares them, and
// hands them to the worker.
void prep_main(mgk_server* S) {
    cudaSetDevice(S->pctx->device);
    for (;;) {
        std::vector<Res> rel;
        std::vector<Job*> fresh;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // the queued request with the most tiles (the earliest on ties) goes first
            auto pick = [&]() -> std::deque<Job*>::iterator {
                auto best = S->queue.begin();
                for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
                    if (tile_count(S, (*it)->req) > tile_count(S, (*best)->req)) best = it;
                return best;
            };
            auto admissible = [&] {
                if (S->queue.empty()) return false;
                const int held = (int)(S->active.size() + S->draining.size()) + S->preparing;
                if (held >= S->max_active) return false;
                return held == 0 || S->reserved + (*pick())->est <= S->budget;
            };
            auto idle = [&] {
                return S->stop && S->queue.empty() && S->preparing == 0 && S->active.empty() &&
                       S->draining.empty() && S->to_release.empty();
            };
            if (S->to_release.empty() && !admissible()) {
                if (idle()) return;
                S->cv_prep.wait_for(lk, std::chrono::milliseconds(50));
            }
            rel.swap(S->to_release);
            while (admissible()) {
                const auto it = pick();
                Job* J = *it;
                S->queue.erase(it);
                J->state = 1;
                J->t_start = Clock::now();
                S->reserved += J->est;
                S->preparing++;
                fresh.push_back(J);
            }
        }
        for (Res& R : rel) release(S->pctx, R);
        for (Job* J : fresh) {
            const int st = prepare(S, J);
            {
                std::lock_guard<std::mutex> lk(S->mu);
                S->preparing--;
                if (st == MGK_OK) {
                    S->active.push_back(J);
                    S->cv_work.notify_one();
                }
            }
            if (st) finish(S, J, st);
        }
    }
}

}  // namespace

extern "C" {

int mgk_serve_create(int device, uint64_t hbm_budget_bytes, int64_t tile_side, int max_active, mgk_server** out) {
    if (!out || max_active <= 0 || tile_side < 64) return MGK_ERR_INVALID;
    *out = nullptr;
    mgk_ctx *c = nullptr, *pc = nullptr;
    int st = mgk_ctx_create(device, hbm_budget_bytes, &c);
    if (st) return st;
    if ((st = mgk_ctx_create(device, hbm_budget_bytes, &pc))) {
        mgk_ctx_destroy(c);
        return st;
    }
    mgk_server* S = new (std::nothrow) mgk_server();
    if (!S) {
        mgk_ctx_destroy(pc);
        mgk_ctx_destroy(c);
        return MGK_ERR_INVALID;
    }
    S->ctx = c;
    S->pctx = pc;
    S->tile = tile_side;
    S->max_active = max_active;
    S->budget = c->budget;
    S->ev_cap = std::max(max_active, kTickTiles);
    if (cudaStreamCreateWithFlags(&S->d2h, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc((void**)&S->h_ev, sizeof(unsigned long long) * (size_t)S->ev_cap, cudaHostAllocMapped) !=
            cudaSuccess ||
        cudaHostGetDevicePointer((void**)&S->d_ev_map, S->h_ev, 0) != cudaSuccess) {
        if (S->h_ev) cudaFreeHost(S->h_ev);
        if (S->d2h) cudaStreamDestroy(S->d2h);
        mgk_ctx_destroy(pc);
        mgk_ctx_destroy(c);
        delete S;
        return MGK_ERR_CUDA;
    }
    S->worker = std::thread(worker_main, S);
    S->prep = std::thread(prep_main, S);
    *out = S;
    return MGK_OK;
}

int mgk_serve_submit(mgk_server* S, const mgk_request* r, uint64_t* ticket) {
    if (!S || !r || !ticket || r->n < 0 || (r->n > 0 && (!r->x || !r->y)) || !(r->h > 0.0f) || !r->out ||
        r->grid.ncols <= 0 || r->grid.nrows <= 0 || !(r->grid.cs > 0.0f) ||
        (r->edge && (!r->edge_mask || r->edge_grid.ncols <= 0 || r->edge_grid.nrows <= 0 || !(r->edge_grid.cs > 0.0f))))
        return MGK_ERR_INVALID;
    Job* J = new (std::nothrow) Job();
    if (!J) return MGK_ERR_INVALID;
    J->req = *r;
    J->est = estimate_bytes(*r, S->tile);
    J->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) {
        delete J;
        return MGK_ERR_INVALID;
    }
    J->id = S->next_id++;
    S->jobs[J->id] = J;
    S->queue.push_back(J);
    *ticket = J->id;
    S->cv_prep.notify_one();
    return MGK_OK;
}

static void fill_result(const Job* J, mgk_result* res) {
    if (!res) return;
    res->status = J->status;
    res->evals = J->evals;
    res->queue_ms = ms_between(J->t_submit, J->t_start);
    res->run_ms = ms_between(J->t_start, J->t_done);
    res->total_ms = ms_between(J->t_submit, J->t_done);
}

int mgk_serve_poll(mgk_server* S, uint64_t ticket, int* done, mgk_result* res) {
    if (!S || !done) return MGK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return MGK_ERR_INVALID;
    Job* J = it->second;
    *done = J->state == 2;
    if (*done) {
        fill_result(J, res);
        S->jobs.erase(it);
        delete J;
    }
    return MGK_OK;
}

int mgk_serve_wait(mgk_server* S, uint64_t ticket, double timeout_s, mgk_result* res) {
    if (!S) return MGK_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->jobs.find(ticket);
    if (it == S->jobs.end()) return MGK_ERR_INVALID;
    Job* J = it->second;
    const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    while (J->state != 2)
        if (S->cv_done.wait_until(lk, until) == std::cv_status::timeout && J->state != 2) return MGK_ERR_TIMEOUT;
    fill_result(J, res);
    S->jobs.erase(ticket);
    const int st = J->status;
    delete J;
    return st;
}

int mgk_serve_stats(mgk_server* S, mgk_serve_info* out) {
    if (!S || !out) return MGK_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    out->ticks = S->ticks;
    out->tiles = S->tiles;
    out->max_batch = S->max_batch;
    out->completed = S->completed;
    out->queued = S->queue.size();
    out->active = S->active.size() + S->draining.size() + (uint64_t)S->preparing;
    out->reserved_bytes = S->reserved;
    out->device_bytes = S->ctx->in_use + S->pctx->in_use;
    return MGK_OK;
}

int mgk_serve_destroy(mgk_server* S) {
    if (!S) return MGK_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
        S->cv_prep.notify_all();
    }
    // both threads finish the queued and active requests first
    if (S->worker.joinable()) S->worker.join();
    if (S->prep.joinable()) S->prep.join();
    for (auto& kv : S->jobs) delete kv.second;
    cudaStreamDestroy(S->d2h);
    cudaFreeHost(S->h_ev);
    mgk_ctx_destroy(S->pctx);
    mgk_ctx_destroy(S->ctx);
    delete S;
    return MGK_OK;
}

}  // extern "C"
