// Autotuner for the index bin side and the streamed tile side.
//
// The reference fixes its launch shapes at compile time (BLOCK_SIZE,
// Utilities.h) and sizes tiles from 20 % of free memory
// (kde_cuda_kdtr_tiled.cu:1186).  Here two sizes are measured on the device
// for the workload at hand:
//  * the bin side of the point index, as a multiple of h: smaller bins give
//    a tighter candidate set per 64 x 64 block but shorter contiguous
//    candidate ranges; each candidate factor is timed on four sample windows
//    of the raster;
//  * the side of streamed density tiles (out-of-core rasters): per-tile
//    planning and launch costs against the pipeline's granularity, timed on
//    the same central area for each candidate side.
// Results are cached in a text file keyed by the GPU, the point count, h in
// cells and the point density, so later runs of a similar workload reuse them
// without measuring again.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "mgk_internal.cuh"

namespace {

double round_sig(double v, int digits) {
    if (!(v > 0.0)) return 0.0;
    const double e = std::floor(std::log10(v)) - (digits - 1);
    const double s = std::pow(10.0, e);
    return std::round(v / s) * s;
}

std::string tune_key(const mgk_ctx* c, const mgk_points* p, float h, const mgk_grid* g) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, c->device);
    std::string name = prop.name;
    for (char& ch : name)
        if (ch == ' ' || ch == '|') ch = '_';
    const double ext = std::max(g->ncols, g->nrows) * (double)g->cs;
    const double rho = (double)p->n * (double)h * (double)h / std::max(ext * ext, 1.0);  // points per h^2
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s|sm%d|n%.2g|hcs%.1g|rho%.1g|side%.1g", name.c_str(), c->sm_count,
                  round_sig((double)p->n, 2), round_sig((double)h / (double)g->cs, 1), round_sig(rho, 1),
                  round_sig((double)std::max(g->ncols, g->nrows), 1));
    return buf;
}

bool cache_lookup(const char* path, const std::string& key, mgk_tuning* t) {
    if (!path) return false;
    FILE* f = std::fopen(path, "r");
    if (!f) return false;
    char k[512];
    float bf, ms;
    int sw;
    long long ts;
    bool found = false;
    while (std::fscanf(f, "%511s %f %d %lld %f", k, &bf, &sw, &ts, &ms) == 5) {
        if (key == k) {  // the last entry for a key wins
            t->bin_factor = bf;
            t->split_waves = sw;
            t->tile_side = ts;
            t->density_ms = ms;
            found = true;
        }
    }
    std::fclose(f);
    return found;
}

void cache_store(const char* path, const std::string& key, const mgk_tuning& t) {
    if (!path) return;
    if (FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %.4f %d %lld %.4f\n", key.c_str(), t.bin_factor, t.split_waves, (long long)t.tile_side,
                     t.density_ms);
        std::fclose(f);
    }
}

}  // namespace

extern "C" {

int mgk_ctx_get_tuning(const mgk_ctx* c, mgk_tuning* t) {
    if (!c || !t) return MGK_ERR_INVALID;
    t->bin_factor = c->bin_factor;
    t->split_waves = c->split_waves;
    t->tile_side = c->tile_side;
    t->density_ms = 0.0f;
    t->from_cache = 0;
    return MGK_OK;
}

int mgk_ctx_set_tuning(mgk_ctx* c, const mgk_tuning* t) {
    if (!c || !t || !(t->bin_factor > 0.0f) || t->split_waves <= 0 || t->tile_side < 0)
        return mgk_fail(c, MGK_ERR_INVALID, "set_tuning: bad values");
    c->bin_factor = t->bin_factor;
    c->split_waves = t->split_waves;
    c->tile_side = t->tile_side;
    return MGK_OK;
}

int mgk_autotune(mgk_ctx* c, const mgk_points* p, float h, const mgk_grid* g, const char* cache_file,
                 mgk_tuning* out) {
    if (!c || !p || !g || !(h > 0.0f) || g->ncols <= 0 || g->nrows <= 0 || !(g->cs > 0.0f))
        return mgk_fail(c, MGK_ERR_INVALID, "autotune: bad arguments");
    mgk_tuning best{};
    mgk_ctx_get_tuning(c, &best);
    const std::string key = tune_key(c, p, h, g);
    if (cache_lookup(cache_file, key, &best)) {
        best.from_cache = 1;
        int st = mgk_ctx_set_tuning(c, &best);
        if (st == MGK_OK && out) *out = best;
        return st;
    }
    // sample windows: four W x W windows around the quarter points of the raster
    const int64_t W = std::min<int64_t>(1024, std::min(g->nrows, g->ncols));
    int64_t win[4][2];
    for (int k = 0; k < 4; k++) {
        const double fr = (k / 2) ? 0.75 : 0.25, fc = (k % 2) ? 0.75 : 0.25;
        win[k][0] = std::min<int64_t>(g->nrows - W, std::max<int64_t>(0, (int64_t)(fr * g->nrows) - W / 2));
        win[k][1] = std::min<int64_t>(g->ncols - W, std::max<int64_t>(0, (int64_t)(fc * g->ncols) - W / 2));
    }
    const int64_t A = std::min<int64_t>(8192, g->nrows), B = std::min<int64_t>(8192, g->ncols);
    float* d_out = nullptr;
    const size_t ob = sizeof(float) * (size_t)A * (size_t)B;
    int st = mgk_alloc(c, (void**)&d_out, std::max(ob, sizeof(float) * (size_t)W * (size_t)W));
    if (st) return st;
    // 1. bin side
    const float factors[4] = {0.5f, 0.75f, 1.0f, 1.25f};
    float best_ms = 1e30f;
    for (float f : factors) {
        if (st) break;
        mgk_index* idx = nullptr;
        if ((st = mgk_index_build(c, p, h, f * h, &idx))) break;
        float ms = 0.0f;
        for (int rep = 0; rep < 2 && st == MGK_OK; rep++) {  // the first pass warms up
            ms = 0.0f;
            for (int k = 0; k < 4 && st == MGK_OK; k++) {
                st = mgk_launch_density(c, idx, g, win[k][0], win[k][1], W, W, nullptr, d_out, nullptr, false);
                ms += c->last_density_ms;
            }
        }
        mgk_index_destroy(idx);
        if (st == MGK_OK && ms < best_ms) {
            best_ms = ms;
            best.bin_factor = f;
        }
    }
    best.density_ms = best_ms;
    // 2. streamed tile side (rasters larger than one 4096 x 4096 tile)
    best.tile_side = 0;
    if (st == MGK_OK && (g->nrows > 4096 || g->ncols > 4096)) {
        mgk_index* idx = nullptr;
        st = mgk_index_build(c, p, h, best.bin_factor * h, &idx);
        const int64_t r0 = (g->nrows - A) / 2, c0 = (g->ncols - B) / 2;
        double best_t = 1e30;
        const int64_t sides[3] = {2048, 4096, 8192};
        for (int64_t T : sides) {
            if (st) break;
            double t_sum = 0.0;
            for (int rep = 0; rep < 2 && st == MGK_OK; rep++) {
                const auto t0 = std::chrono::steady_clock::now();
                for (int64_t r = 0; r < A && st == MGK_OK; r += T)
                    for (int64_t q = 0; q < B && st == MGK_OK; q += T)
                        st = mgk_launch_density(c, idx, g, r0 + r, c0 + q, std::min(T, A - r), std::min(T, B - q),
                                                nullptr, d_out, nullptr, false);
                t_sum = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            }
            if (st == MGK_OK && t_sum < best_t) {
                best_t = t_sum;
                best.tile_side = T;
            }
        }
        mgk_index_destroy(idx);
    }
    mgk_free(c, d_out, std::max(ob, sizeof(float) * (size_t)W * (size_t)W));
    if (st) return st;
    best.from_cache = 0;
    if ((st = mgk_ctx_set_tuning(c, &best))) return st;
    cache_store(cache_file, key, best);
    if (out) *out = best;
    return MGK_OK;
}

}  // extern "C"
