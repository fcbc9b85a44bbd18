// mgkde_tiled: host driver with the reference's command line (main(),
// kde_cuda_kdtr_tiled.cu:262-1560), running the GPU path on one B200 through
// the C ABI (libmgk.so).
//
//   mode 0: mgkde_tiled 0 #points cellsize_edge_correction cellsize_density h_option
//           enable_edge_correction enable_sample_weight skip_omp_parallel skip_gpu_parallel
//           num_cpu_threads num_gpu denfn_seq denfn_cuda serialized_mode [--key=value ...]
//   mode 1: mgkde_tiled 1 points_file mask_file_edge_correction mask_file_density h_option ...
//
// The 14 positional arguments keep their meaning.  h_option: 0 rule of thumb,
// 1 leave-one-out maximum likelihood (golden section), -1 per-point h from
// the CSV, 2 adaptive bandwidths (Hooke-Jeeves over h0 and alpha).
// The OpenMP CPU path (skip_omp_parallel = 0) is not part of this build: only
// the GPU path runs and writes denfn_cuda and pntsCUDA.csv.  num_gpu > 1 runs
// on one GPU (this build is single-GPU; tiles need no exchange).
// serialized_mode must be 0 (the reference's author advises 0).
// Extras: --device=D  --tile=N (tile side, cells)  --bin=S (index bin side)
//         --h=H (fixed bandwidth, overrides h_option 0)  --budget=BYTES
//         --resume (skip the density tiles listed in <denfn_cuda>.tiles by an
//         interrupted run and write the rest into its GeoTIFF)
//         --max-tiles=K (write at most K density tiles, then stop with exit
//         code 2 so that a later --resume run continues: work in time slices)
//         --autotune[=CACHE_FILE] (measure the index bin side and the density
//         tile side for this workload first; fixed h only)
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mgk.h"
#include "tiff_io.hpp"

namespace {

using Clock = std::chrono::high_resolution_clock;
double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

struct Args {
    int mode = 0;
    int npts = 100;
    float cs_edge = 1.0f, cs_density = 0.5f;
    std::string pnt_fn, mask_fn, mask_density_fn;
    int hoption = 0;
    bool edge = false, sample_weights = false;
    int skip_omp = 0, skip_gpu = 0, threads = 1, ngpu = 1;
    std::string den_omp_fn, den_cuda_fn;
    int serialized = 0;
    int device = 0;
    int64_t tile = 0;
    float bin = 0.0f;
    float h_fixed = 0.0f;
    uint64_t budget = 0;
    bool resume = false;
    int64_t max_tiles = -1;
    bool autotune = false;
    std::string tune_cache;
};

void usage() {
    std::printf(
        "Run in mode 0:\n mgkde_tiled 0 #points cellsize_edge_correction cellsize_density h_option "
        "enable_edge_corection enable_sample_weight skip_omp_parallel skip_gpu_parallel num_cpu_threads num_gpu "
        "denfn_omp denfn_cuda serialized_mode\n"
        "Run in mode 1:\n mgkde_tiled 1 points_file mask_file_edge_correction mask_file_density h_option "
        "enable_edge_corection enable_sample_weight skip_omp_parallel skip_gpu_parallel num_cpu_threads num_gpu "
        "denfn_omp denfn_cuda serialized_mode\n");
}

bool parse(int argc, char** argv, Args& a) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; i++) {
        std::string s = argv[i];
        if (s.rfind("--", 0) == 0) {
            auto eq = s.find('=');
            std::string k = s.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
            std::string v = eq == std::string::npos ? "" : s.substr(eq + 1);
            if (k == "device") a.device = std::atoi(v.c_str());
            else if (k == "tile") a.tile = std::atoll(v.c_str());
            else if (k == "bin") a.bin = (float)std::atof(v.c_str());
            else if (k == "h") a.h_fixed = (float)std::atof(v.c_str());
            else if (k == "budget") a.budget = std::strtoull(v.c_str(), nullptr, 10);
            else if (k == "resume") a.resume = true;
            else if (k == "max-tiles") a.max_tiles = std::atoll(v.c_str());
            else if (k == "autotune") { a.autotune = true; a.tune_cache = v; }
            else { std::printf("***Unknown option %s\n", s.c_str()); return false; }
        } else {
            pos.push_back(s);
        }
    }
    if (pos.size() != 14) return false;
    a.mode = std::atoi(pos[0].c_str());
    if (a.mode == 0) {
        a.npts = std::atoi(pos[1].c_str());
        a.cs_edge = (float)std::atof(pos[2].c_str());
        a.cs_density = (float)std::atof(pos[3].c_str());
    } else if (a.mode == 1) {
        a.pnt_fn = pos[1];
        a.mask_fn = pos[2];
        a.mask_density_fn = pos[3];
    } else {
        return false;
    }
    a.hoption = std::atoi(pos[4].c_str());
    a.edge = std::atoi(pos[5].c_str()) != 0;
    a.sample_weights = std::atoi(pos[6].c_str()) != 0;
    a.skip_omp = std::atoi(pos[7].c_str());
    a.skip_gpu = std::atoi(pos[8].c_str());
    a.threads = std::atoi(pos[9].c_str());
    a.ngpu = std::atoi(pos[10].c_str());
    a.den_omp_fn = pos[11];
    a.den_cuda_fn = pos[12];
    a.serialized = std::atoi(pos[13].c_str());
    return true;
}

// ReadSamplePoints (kde_cuda_kdtr_tiled.cu:1623-1711): header skipped,
// x,y[,h],w; weights used only with enable_sample_weight.
bool read_points(const Args& a, std::vector<float>& x, std::vector<float>& y, std::vector<float>& w,
                 std::vector<float>& h) {
    FILE* f = std::fopen(a.pnt_fn.c_str(), "rt");
    if (!f) {
        std::printf("***Error opening file %s\n", a.pnt_fn.c_str());
        return false;
    }
    char line[4096];
    if (!std::fgets(line, sizeof(line), f)) {
        std::fclose(f);
        std::printf("***No point in file!\n");
        return false;
    }
    while (std::fgets(line, sizeof(line), f)) {
        std::vector<float> v;
        for (char* t = std::strtok(line, ",\n\r"); t; t = std::strtok(nullptr, ",\n\r")) v.push_back((float)std::atof(t));
        if (v.empty()) continue;
        const size_t need = a.hoption == -1 ? 4 : 3;
        if (v.size() < need - (a.hoption == -1 ? 0 : 1)) {
            std::printf("***Error - malformed line in %s\n", a.pnt_fn.c_str());
            std::fclose(f);
            return false;
        }
        x.push_back(v[0]);
        y.push_back(v[1]);
        if (a.hoption == -1) {
            if (v.size() < 4) {
                std::printf("***Error - No bandwidth provided in the file\n");
                std::fclose(f);
                return false;
            }
            h.push_back(v[2]);
            w.push_back(a.sample_weights ? v[3] : 1.0f);
        } else {
            w.push_back(a.sample_weights && v.size() > 2 ? v[2] : 1.0f);
        }
    }
    std::fclose(f);
    if (x.empty()) {
        std::printf("***No point in file!\n");
        return false;
    }
    return true;
}

int check(mgk_ctx* ctx, int st, const char* what) {
    if (st != MGK_OK) std::printf("***%s failed: %s (%s)\n", what, mgk_status_string(st), mgk_ctx_last_error(ctx));
    return st;
}

}  // namespace

int main(int argc, char** argv) {
    const auto T1 = Clock::now();
    Args a;
    if (!parse(argc, argv, a)) {
        std::printf("Incorrect arguments provided. Exiting...\n");
        usage();
        return 1;
    }
    if (a.mode == 0 && a.hoption == -1) {
        std::printf("***Error - should never use bandwidth option -1 in mode 0 (i.e., randomly generately points). Exiting...");
        return 1;
    }
    if (a.hoption < -1 || a.hoption > 2) {
        std::printf("***Error - unknown h_option %d\n", a.hoption);
        return 1;
    }
    if (a.serialized != 0) std::printf("===serialized_mode is ignored (always 0 in this build)\n");
    if (a.skip_omp == 0) std::printf("===The OpenMP CPU path is not part of this build; running the GPU path only\n");
    if (a.skip_gpu != 0) {
        std::printf("===skip_gpu_parallel=1: nothing to run\n");
        return 0;
    }
    if (a.ngpu > 1) std::printf("===This build runs on one GPU (device %d)\n", a.device);

    // ---- inputs ---------------------------------------------------------
    std::vector<float> x, y, w, hpp;
    mgk_grid eg{}, dg{};
    std::vector<float> emask, dmask;
    double dens_gt[6];
    bool dmask_all_valid = false;
    auto t1 = Clock::now();
    if (a.mode == 1) {
        if (!read_points(a, x, y, w, hpp)) return 1;
        mgk_tiff::Raster r, rd;
        std::string err;
        if (!mgk_tiff::read_tiff(a.mask_fn, r, err)) { std::printf("***%s\n", err.c_str()); return 1; }
        if (!mgk_tiff::read_tiff(a.mask_density_fn, rd, err)) { std::printf("***%s\n", err.c_str()); return 1; }
        // ReadGeoTIFFRaster (kde_cuda_kdtr_tiled.cu:2040-2080)
        eg = {r.ncols, r.nrows, (float)r.gt[0], (float)(r.gt[3] + r.nrows * r.gt[5]), (float)r.gt[1],
              (float)(r.has_nodata ? r.nodata : -1e10)};
        emask.swap(r.data);
        dg = {rd.ncols, rd.nrows, (float)rd.gt[0], (float)(rd.gt[3] + rd.nrows * rd.gt[5]), (float)rd.gt[1],
              (float)(rd.has_nodata ? rd.nodata : -1e10)};
        dmask.swap(rd.data);
        std::memcpy(dens_gt, rd.gt, sizeof(dens_gt));
    } else {
        // AllocateSamplePoints (:1598-1620) with srand(100) (:407)
        std::srand(100);
        for (int i = 0; i < a.npts; i++) {
            x.push_back(std::rand() * 100.0f / RAND_MAX);
            y.push_back(std::rand() * 100.0f / RAND_MAX);
            w.push_back(1.0f);
        }
        const int n_e = int(100 / a.cs_edge);
        eg = {n_e, n_e, 0.0f, 0.0f, a.cs_edge, -9999.0f};
        emask.assign((size_t)n_e * n_e, 0.0f);
        const int n_d = int(std::ceil(100.0 / a.cs_density));
        dg = {n_d, n_d, 0.0f, 100.0f - n_d * a.cs_density, a.cs_density, -9999.0f};
        dmask_all_valid = true;
        const double gt[6] = {0, a.cs_density, 0, 100.0, 0, -1.0 * a.cs_density};
        std::memcpy(dens_gt, gt, sizeof(gt));
    }
    const int64_t n = (int64_t)x.size();
    std::printf("...reading in data took %.0f ms\n", ms_since(t1));
    std::printf("===Number of points: %lld\n", (long long)n);
    std::printf("===Cell size (edge correction): %f\n", eg.cs);
    std::printf("===Number of cells (edge correction): %lld\n", (long long)(eg.ncols * eg.nrows));
    std::printf("===Cell size (density estimation): %f\n", dg.cs);
    std::printf("===Number of cells (density estimation): %lld\n", (long long)(dg.ncols * dg.nrows));
    std::printf("===Bandwidth option: %d\n===Enable edge correction: %d\n===Enable sample weight: %d\n", a.hoption,
                (int)a.edge, (int)a.sample_weights);

    float h = mgk_rule_of_thumb(n, x.data(), y.data(), w.data());
    std::printf("===Rule of thumb bandwidth h0: %.5f\n", h);
    if (a.h_fixed > 0.0f) h = a.h_fixed;

    mgk_ctx* ctx = nullptr;
    int st = mgk_ctx_create(a.device, a.budget, &ctx);
    if (st != MGK_OK) {
        std::printf("***No usable B200 device (%s)\n", mgk_status_string(st));
        return 1;
    }
    const auto t_gpu = Clock::now();
    mgk_points* pts = nullptr;
    mgk_raster* em = nullptr;
    mgk_index* idx = nullptr;
    int rc = 1;
    do {
        if (check(ctx, mgk_points_upload(ctx, n, x.data(), y.data(), w.data(), hpp.empty() ? nullptr : hpp.data(), &pts),
                  "points upload")) break;
        const float hcall = a.hoption == -1 ? 0.0f : h;
        if (a.edge) {
            if (check(ctx, mgk_raster_upload(ctx, &eg, emask.data(), &em), "mask upload")) break;
            t1 = Clock::now();
            if (check(ctx, mgk_boundary_dist(ctx, pts, em), "boundary distance")) break;
            mgk_ctx_synchronize(ctx);
            std::printf("...MarkBoundary + CalcDist2Boundary took %.0f ms\n", ms_since(t1));
        }
        if (a.hoption == 1) {
            float hopt = h;
            int it = 0;
            t1 = Clock::now();
            if (check(ctx, mgk_mle_fixed_bandwidth(ctx, pts, em, h, &hopt, &it), "bandwidth search")) break;
            std::printf("cross validated optimal fixed bandwidth hopt: %.5f (%d iterations, %.0f ms)\n", hopt, it,
                        ms_since(t1));
            h = hopt;
        }
        if (a.hoption == 2) {  // adaptive bandwidths (main, kde_cuda_kdtr_tiled.cu:548-573)
            float hopt = h, aopt = -0.5f;
            double lmax = 0.0;
            int it = 0;
            hpp.assign((size_t)n, 0.0f);
            t1 = Clock::now();
            if (check(ctx, mgk_adaptive_bandwidths(ctx, pts, em, h, &hopt, &aopt, &lmax, &it, hpp.data()),
                      "adaptive bandwidth search"))
                break;
            std::printf("h0: %.5f alpha0: %.5f Lmax: %.5f (%d iterations, %.0f ms)\n", hopt, aopt, lmax, it,
                        ms_since(t1));
            h = hopt;
        }
        const float hfinal = (a.hoption == -1 || a.hoption == 2) ? 0.0f : h;
        (void)hcall;
        t1 = Clock::now();
        if (a.edge) {
            if (check(ctx, mgk_edge_weights(ctx, pts, em, hfinal, nullptr), "edge weights")) break;
        } else {
            if (check(ctx, mgk_edge_weights_unit(ctx, pts), "unit weights")) break;
        }
        mgk_ctx_synchronize(ctx);
        std::printf("...CalcEdgeCorrectionWeights took %.0f ms\n", ms_since(t1));
        mgk_tuning tuned{};
        bool have_tuning = false;
        if (a.autotune && hpp.empty()) {
            t1 = Clock::now();
            if (check(ctx, mgk_autotune(ctx, pts, hfinal, &dg, a.tune_cache.empty() ? nullptr : a.tune_cache.c_str(),
                                        &tuned), "autotune"))
                break;
            have_tuning = true;
            std::printf("...autotune: bin side %.2f h, tile side %lld%s (%.0f ms)\n", tuned.bin_factor,
                        (long long)tuned.tile_side, tuned.from_cache ? " (cached)" : "", ms_since(t1));
        }
        if (check(ctx, mgk_index_build(ctx, pts, hfinal, a.bin, &idx), "index build")) break;

        // ---- tiled density (kde_cuda_kdtr_tiled.cu:1146-1517) ----------
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        int64_t T = a.tile;
        if (T <= 0 && have_tuning && tuned.tile_side > 0) T = tuned.tile_side;
        if (T <= 0) {  // largest square tile whose mask + output fit in 20% of free memory
            const double cells = 0.2 * (double)fr / 8.0;
            T = (int64_t)std::sqrt(cells);
            T = std::max<int64_t>(256, T / 256 * 256);
        }
        const int64_t tr = std::min<int64_t>(T, dg.nrows), tc = std::min<int64_t>(T, dg.ncols);
        std::printf("...TILE_XSIZE=%lld, TILE_YSIZE=%lld\n", (long long)tc, (long long)tr);
        // Completed tiles are appended to <output>.tiles after their data is
        // written, so --resume can skip them after an interruption.
        const int64_t ntx = (dg.ncols + tc - 1) / tc, nty = (dg.nrows + tr - 1) / tr;
        std::vector<uint8_t> done((size_t)(ntx * nty), 0);
        const std::string log_fn = a.den_cuda_fn + ".tiles";
        bool resuming = false;
        if (a.resume) {
            if (FILE* lf = std::fopen(log_fn.c_str(), "r")) {
                long long t = 0;
                while (std::fscanf(lf, "%lld", &t) == 1)
                    if (t >= 0 && t < ntx * nty) done[(size_t)t] = 1;
                std::fclose(lf);
                resuming = true;
            }
        }
        mgk_tiff::TiledWriter wr;
        if (!wr.open(a.den_cuda_fn, dg.ncols, dg.nrows, dens_gt, true, dg.nodata, 256, 0.0f, resuming)) {
            std::printf("***Cannot create %s\n", a.den_cuda_fn.c_str());
            break;
        }
        FILE* tile_log = std::fopen(log_fn.c_str(), resuming ? "a" : "w");
        struct Sink {
            mgk_tiff::TiledWriter* wr;
            FILE* log;
            int64_t max_tiles;
            int64_t n = 0;
        } sk{&wr, tile_log, a.max_tiles};
        auto sink = [](void* u, int64_t t, int64_t r0, int64_t c0, int64_t nr, int64_t nc, const float* d) -> int {
            Sink* s = static_cast<Sink*>(u);
            if (s->max_tiles >= 0 && s->n >= s->max_tiles) return 1;  // this run's tile allowance is used up
            if (!s->wr->write_region(c0, r0, nc, nr, d) || !s->wr->flush()) return 1;
            if (s->log) {
                std::fprintf(s->log, "%lld\n", (long long)t);
                std::fflush(s->log);
            }
            std::printf("...wrote tile %lld: rows %lld+%lld cols %lld+%lld\n", (long long)t, (long long)r0,
                        (long long)nr, (long long)c0, (long long)nc);
            s->n++;
            return 0;
        };
        struct Src {
            const float* mask;
            int64_t ncols;
        } src{dmask_all_valid ? nullptr : dmask.data(), dg.ncols};
        auto source = [](void* u, int64_t, int64_t r0, int64_t c0, int64_t nr, int64_t nc, float* out) -> int {
            const Src* s = static_cast<const Src*>(u);
            for (int64_t r = 0; r < nr; r++)
                std::memcpy(out + r * nc, s->mask + (r0 + r) * s->ncols + c0, sizeof(float) * nc);
            return 0;
        };
        t1 = Clock::now();
        int64_t evals_total = 0;
        const int dst = mgk_density_stream(ctx, idx, &dg, T, dmask_all_valid ? nullptr : +source,
                                           &src, +sink, &sk, done.data(), &evals_total);
        if (tile_log) std::fclose(tile_log);
        wr.close();
        if (dst != MGK_OK) {
            if (dst == MGK_ERR_IO && a.max_tiles >= 0 && sk.n >= a.max_tiles) {
                std::printf("...stopped after %lld tiles (--max-tiles); rerun with --resume to continue\n",
                            (long long)sk.n);
                rc = 2;
            } else {
                std::printf("***density: %s (%s); rerun with --resume to continue\n", mgk_status_string(dst),
                            mgk_ctx_last_error(ctx));
            }
            break;
        }
        std::remove(log_fn.c_str());  // complete: nothing to resume
        std::printf("KernelDensityEstimation took %.0f ms (%lld kernel evaluations)\n", ms_since(t1),
                    (long long)evals_total);

        // WriteSamplePoints (kde_cuda_kdtr_tiled.cu:1857-1870): x, y, h, edge weight (input order)
        std::vector<float> ew(n);
        if (check(ctx, mgk_points_download(pts, nullptr, ew.data()), "download")) break;
        FILE* f = std::fopen("pntsCUDA.csv", "w");
        if (f) {
            std::fprintf(f, "x, y, h, w\n");
            for (int64_t i = 0; i < n; i++)
                std::fprintf(f, "%f, %f, %f, %f\n", x[i], y[i], hpp.empty() ? h : hpp[i], ew[i]);
            std::fclose(f);
        }
        std::printf("\n>>>>>>Computation on GPU took %.0f ms in total\n\n", ms_since(t_gpu));
        rc = 0;
    } while (0);
    mgk_index_destroy(idx);
    mgk_raster_destroy(em);
    mgk_points_destroy(pts);
    mgk_ctx_destroy(ctx);
    std::printf("Done...\n\n+++In total it took %.0f ms\n", ms_since(T1));
    return rc;
}
