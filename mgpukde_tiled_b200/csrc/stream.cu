// Out-of-core tile pipeline: a raster larger than the host wants to hold,
// produced tile by tile and handed to a sink (a GeoTIFF writer, a file, a
// host array) while the GPU computes the next tiles.
//
// The reference walks the tiles in row-major order and for each one reads
// the mask tile, computes, copies back and writes it, all in sequence
// (kde_cuda_kdtr_tiled.cu:1233-1517 with GeoTIFF.cpp:494-575).  Here:
//  * the mask tile (when a source is given) is read on the calling thread
//    into a pinned buffer and copied to the device on a copy stream;
//  * the density of tile k runs on the context stream;
//  * its result is copied to one of three pinned host buffers on the copy
//    stream, and a writer thread hands finished tiles to the sink in order,
//    so disk writes overlap the next tiles' compute and copies;
//  * tiles marked in `done` (a resume after an interrupted run) are skipped,
//    and the sink is told about each tile only after its data is final, so a
//    caller that records completed tiles can restart where it stopped.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "mgk_internal.cuh"

// device result buffers in flight: tile k computes into buffer k % kOutBufs
// while the copies of the tiles before it leave
#ifndef MGK_STREAM_OUT_BUFS
#define MGK_STREAM_OUT_BUFS 3
#endif
constexpr int kOutBufs = MGK_STREAM_OUT_BUFS;
static_assert(kOutBufs >= 2 && kOutBufs <= 3, "the copy slots are three");

namespace {

struct Slot {
    float* host = nullptr;  // pinned
    int64_t tile = -1, r0 = 0, c0 = 0, nr = 0, nc = 0;
    cudaEvent_t copied = nullptr;
    bool busy = false;  // queued for, or in, the sink
};

struct Writer {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Slot*> q;
    bool stop = false;
    int status = MGK_OK;
    mgk_tile_sink sink = nullptr;
    void* user = nullptr;
    int device = 0;

    void run() {
        cudaSetDevice(device);
        for (;;) {
            Slot* s = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !q.empty(); });
                if (q.empty()) return;
                s = q.front();
            }
            int st = MGK_OK;
            if (cudaEventSynchronize(s->copied) != cudaSuccess) st = MGK_ERR_CUDA;
            if (st == MGK_OK && status == MGK_OK && sink(user, s->tile, s->r0, s->c0, s->nr, s->nc, s->host) != 0)
                st = MGK_ERR_IO;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (st && status == MGK_OK) status = st;
                q.pop_front();
                s->busy = false;
            }
            cv.notify_all();
        }
    }
};

}  // namespace

extern "C" int mgk_density_stream(mgk_ctx* c, const mgk_index* idx, const mgk_grid* g, int64_t tile_side,
                                  mgk_tile_source mask_src, void* src_user, mgk_tile_sink sink, void* sink_user,
                                  const uint8_t* done, int64_t* evals) {
    if (!c || !idx || !g || g->ncols <= 0 || g->nrows <= 0 || !(g->cs > 0.0f) || !sink || tile_side <= 0)
        return mgk_fail(c, MGK_ERR_INVALID, "density_stream: bad arguments");
    cudaSetDevice(c->device);
    const int64_t tr = std::min<int64_t>(tile_side, g->nrows), tc = std::min<int64_t>(tile_side, g->ncols);
    const int64_t ntx = (g->ncols + tc - 1) / tc, nty = (g->nrows + tr - 1) / tr;
    const size_t tb = sizeof(float) * (size_t)tr * (size_t)tc;
    cudaStream_t cs = nullptr;
    float *d_out[kOutBufs] = {}, *d_mask = nullptr, *h_mask = nullptr;
    cudaEvent_t ev_den[kOutBufs] = {}, ev_mask = nullptr;
    Slot slots[3];
    unsigned long long* d_ev = nullptr;
    int st = MGK_OK;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return mgk_fail(c, MGK_ERR_CUDA, "stream");
    for (int b = 0; b < kOutBufs && st == MGK_OK; b++) {
        st = mgk_alloc(c, (void**)&d_out[b], tb);
        if (st == MGK_OK && cudaEventCreateWithFlags(&ev_den[b], cudaEventDisableTiming) != cudaSuccess)
            st = mgk_fail(c, MGK_ERR_CUDA, "event");
    }
    if (st == MGK_OK && mask_src) {
        st = mgk_alloc(c, (void**)&d_mask, tb);
        if (st == MGK_OK && cudaMallocHost((void**)&h_mask, tb) != cudaSuccess) st = mgk_fail(c, MGK_ERR_CUDA, "pinned");
        if (st == MGK_OK && cudaEventCreateWithFlags(&ev_mask, cudaEventDisableTiming) != cudaSuccess)
            st = mgk_fail(c, MGK_ERR_CUDA, "event");
    }
    // The library's own copy sink into page-locked host memory: the result
    // tiles are copied straight into the target raster (2-D copies on the
    // copy stream), without the staging buffers and the writer thread.
    const mgk_copy_target* direct = nullptr;
    if (sink == mgk_copy_sink && sink_user) {
        const mgk_copy_target* t = static_cast<const mgk_copy_target*>(sink_user);
        cudaPointerAttributes pa{};
        if (t->base && cudaPointerGetAttributes(&pa, t->base) == cudaSuccess && pa.type == cudaMemoryTypeHost)
            direct = t;
        cudaGetLastError();
    }
    // three page-locked staging tiles for the writer thread (not needed by the
    // direct copies; pinning them costs tens of ms for 4096^2 tiles)
    for (int b = 0; b < 3 && st == MGK_OK; b++) {
        if (!direct && cudaMallocHost((void**)&slots[b].host, tb) != cudaSuccess)
            st = mgk_fail(c, MGK_ERR_CUDA, "pinned");
        else if (cudaEventCreateWithFlags(&slots[b].copied, cudaEventDisableTiming) != cudaSuccess)
            st = mgk_fail(c, MGK_ERR_CUDA, "event");
    }
    if (st == MGK_OK && evals) {
        st = mgk_alloc(c, (void**)&d_ev, sizeof(unsigned long long));
        if (st == MGK_OK && cudaMemsetAsync(d_ev, 0, sizeof(unsigned long long), c->stream) != cudaSuccess)
            st = MGK_ERR_CUDA;
    }
    Writer W;
    W.sink = sink;
    W.user = sink_user;
    W.device = c->device;
    std::thread wt;
    if (st == MGK_OK) wt = std::thread([&W] { W.run(); });
    // The tiles this call computes (a resume skips those marked done).
    std::vector<int64_t> todo;
    for (int64_t t = 0; t < ntx * nty; t++)
        if (!done || !done[t]) todo.push_back(t);
    auto geom = [&](int64_t t, int64_t& r0, int64_t& c0, int64_t& nr, int64_t& nc) {
        r0 = (t / ntx) * tr;
        c0 = (t % ntx) * tc;
        nr = std::min(tr, g->nrows - r0);
        nc = std::min(tc, g->ncols - c0);
    };
    // Tile k + 1 is planned while tile k computes: its counting kernel is
    // queued on the context stream ahead of tile k's density, the host plans
    // from the counts (staging slot 1 + (k + 1) % 2) while that density runs,
    // and the next launch follows without a gap.  The staging-wait flag
    // (counter 7) is shared by all tiles: zeroed here, read at the end.
    mgk_dplan* plans[2] = {nullptr, nullptr};
    cudaEvent_t counted = nullptr;
    if (st == MGK_OK && cudaEventCreateWithFlags(&counted, cudaEventDisableTiming) != cudaSuccess)
        st = mgk_fail(c, MGK_ERR_CUDA, "event");
    if (st == MGK_OK && cudaMemsetAsync(c->d_counter + 7, 0, sizeof(unsigned long long), c->stream) != cudaSuccess)
        st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: flag");
    for (int i = 1; i <= 2 && st == MGK_OK; i++) {  // slots sized for a full tile up front
        void *hs = nullptr, *ds = nullptr;
        st = mgk_host_stage_slot(c, i, 64 * (size_t)((tr + 63) / 64) * (size_t)((tc + 127) / 128) + 4096, &hs, &ds);
    }
    auto count_of = [&](size_t k) -> int {
        int64_t r0, c0, nr, nc;
        geom(todo[k], r0, c0, nr, nc);
        return mgk_density_counts_launch(c, idx, g, r0, c0, nr, nc, 1 + (int)(k & 1), c->stream);
    };
    auto plan_of = [&](size_t k) -> int {  // after tile k's counting kernel has finished
        int64_t r0, c0, nr, nc;
        geom(todo[k], r0, c0, nr, nc);
        const int b = (int)(k & 1);
        mgk_density_discard(c, plans[b]);  // tile k - 2's, whose kernels have ended
        plans[b] = nullptr;
        return mgk_density_plan_counted(c, idx, g, r0, c0, nr, nc, mask_src ? d_mask : nullptr, d_out[k % kOutBufs], d_ev,
                                        1 + b, &plans[b]);
    };
    if (st == MGK_OK && !todo.empty() && (st = count_of(0)) == MGK_OK) {
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: plan");
        else st = plan_of(0);
    }
    for (size_t k_out = 0; st == MGK_OK && k_out < todo.size(); k_out++) {
        const int64_t t = todo[k_out];
        {
            std::lock_guard<std::mutex> lk(W.mu);
            if (W.status) {
                st = W.status;
                break;
            }
        }
        int64_t r0, c0, nr, nc;
        geom(t, r0, c0, nr, nc);
        const int b = (int)(k_out % kOutBufs);
        // the mask tile: read on this thread, copied on the copy stream
        if (mask_src) {
            if (ev_mask && cudaEventSynchronize(ev_mask) != cudaSuccess) { st = MGK_ERR_CUDA; break; }
            if (mask_src(src_user, t, r0, c0, nr, nc, h_mask) != 0) {
                st = mgk_fail(c, MGK_ERR_IO, "density_stream: the mask source failed");
                break;
            }
            // the previous density must be done with d_mask before it is overwritten
            if (cudaStreamWaitEvent(cs, ev_den[(b + kOutBufs - 1) % kOutBufs], 0) != cudaSuccess ||
                cudaMemcpyAsync(d_mask, h_mask, sizeof(float) * nr * nc, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
                cudaEventRecord(ev_mask, cs) != cudaSuccess) {
                st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: mask copy");
                break;
            }
        }
        // the next tile's counting kernel goes ahead of this tile's density
        if (k_out + 1 < todo.size()) {
            if ((st = count_of(k_out + 1))) break;
            if (cudaEventRecord(counted, c->stream) != cudaSuccess) { st = MGK_ERR_CUDA; break; }
        }
        if (mask_src && cudaStreamWaitEvent(c->stream, ev_mask, 0) != cudaSuccess) { st = MGK_ERR_CUDA; break; }
        // d_out[b] was last copied out kOutBufs tiles ago
        if (k_out >= (size_t)kOutBufs && cudaStreamWaitEvent(c->stream, slots[(k_out - kOutBufs) % 3].copied, 0) != cudaSuccess) {
            st = MGK_ERR_CUDA;
            break;
        }
        if ((st = mgk_density_launch_plan(c, plans[k_out & 1], c->stream))) break;
        if (cudaEventRecord(ev_den[b], c->stream) != cudaSuccess) { st = MGK_ERR_CUDA; break; }
        if (direct) {
            if (cudaStreamWaitEvent(cs, ev_den[b], 0) != cudaSuccess ||
                cudaMemcpy2DAsync(direct->base + r0 * direct->ncols + c0, sizeof(float) * direct->ncols, d_out[b],
                                  sizeof(float) * nc, sizeof(float) * nc, nr, cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
                cudaEventRecord(slots[k_out % 3].copied, cs) != cudaSuccess) {
                st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: result copy");
                break;
            }
        } else {
            // a free host slot (the writer may still hold the one used three tiles ago)
            Slot* sl = &slots[k_out % 3];
            {
                std::unique_lock<std::mutex> lk(W.mu);
                W.cv.wait(lk, [&] { return !sl->busy || W.status != MGK_OK; });
                if (W.status) { st = W.status; break; }
            }
            sl->tile = t;
            sl->r0 = r0;
            sl->c0 = c0;
            sl->nr = nr;
            sl->nc = nc;
            if (cudaStreamWaitEvent(cs, ev_den[b], 0) != cudaSuccess ||
                cudaMemcpyAsync(sl->host, d_out[b], sizeof(float) * nr * nc, cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
                cudaEventRecord(sl->copied, cs) != cudaSuccess) {
                st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: result copy");
                break;
            }
            {
                std::lock_guard<std::mutex> lk(W.mu);
                sl->busy = true;
                W.q.push_back(sl);
            }
            W.cv.notify_all();
        }
        if (k_out + 1 < todo.size()) {
            if (cudaEventSynchronize(counted) != cudaSuccess) { st = mgk_fail(c, MGK_ERR_CUDA, "density_stream: plan"); break; }
            st = plan_of(k_out + 1);
        }
    }
    if (wt.joinable()) {
        {
            std::lock_guard<std::mutex> lk(W.mu);
            W.stop = true;
        }
        W.cv.notify_all();
        wt.join();  // drains the queued tiles (the sink is skipped once it has failed)
        if (st == MGK_OK) st = W.status;
        if (st == MGK_ERR_IO && W.status == MGK_ERR_IO) mgk_fail(c, MGK_ERR_IO, "density_stream: the tile sink failed");
    }
    cudaStreamSynchronize(c->stream);
    cudaStreamSynchronize(cs);
    for (int i = 0; i < 2; i++) mgk_density_discard(c, plans[i]);  // every kernel has ended
    if (counted) cudaEventDestroy(counted);
    if (st == MGK_OK) {
        unsigned long long flag = 0;
        if (cudaMemcpy(&flag, c->d_counter + 7, sizeof(flag), cudaMemcpyDeviceToHost) != cudaSuccess) st = MGK_ERR_CUDA;
        else if (flag) st = mgk_fail(c, MGK_ERR_TIMEOUT, "density: a shared-memory staging wait timed out");
    }
    if (st == MGK_OK && evals) {
        unsigned long long v = 0;
        if (cudaMemcpy(&v, d_ev, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) st = MGK_ERR_CUDA;
        *evals = (int64_t)v;
    }
    for (int b = 0; b < kOutBufs; b++) {
        mgk_free(c, d_out[b], tb);
        if (ev_den[b]) cudaEventDestroy(ev_den[b]);
    }
    mgk_free(c, d_mask, tb);
    mgk_free(c, d_ev, sizeof(unsigned long long));
    if (h_mask) cudaFreeHost(h_mask);
    if (ev_mask) cudaEventDestroy(ev_mask);
    for (auto& s : slots) {
        if (s.host) cudaFreeHost(s.host);
        if (s.copied) cudaEventDestroy(s.copied);
    }
    cudaStreamDestroy(cs);
    return st;
}

extern "C" int mgk_copy_sink(void* target, int64_t, int64_t r0, int64_t c0, int64_t nr, int64_t nc,
                             const float* d) {
    const mgk_copy_target* t = static_cast<const mgk_copy_target*>(target);
    if (!t || !t->base) return 1;
    for (int64_t r = 0; r < nr; r++)
        std::memcpy(t->base + (r0 + r) * t->ncols + c0, d + r * nc, sizeof(float) * (size_t)nc);
    return 0;
}
