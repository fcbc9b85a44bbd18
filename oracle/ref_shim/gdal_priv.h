/*
 * Test infrastructure: a small stand-in for the part of GDAL's C++ API that
 * the reference's GeoTIFF.cpp uses, so the reference program can be built
 * here from its own sources (oracle/ref_build.sh) without GDAL.  Reading and
 * writing go through the project's header-only TIFF codec (tiff_io.hpp).
 * Only band 1, Float32 output, and the calls GeoTIFF.cpp makes exist.
 */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cmath>
#include <algorithm>

#include "tiff_io.hpp"

typedef enum { CE_None = 0, CE_Debug = 1, CE_Warning = 2, CE_Failure = 3, CE_Fatal = 4 } CPLErr;
typedef enum { GA_ReadOnly = 0, GA_Update = 1 } GDALAccess;
typedef enum { GF_Read = 0, GF_Write = 1 } GDALRWFlag;
typedef enum {
    GDT_Unknown = 0, GDT_Byte = 1, GDT_UInt16 = 2, GDT_Int16 = 3, GDT_UInt32 = 4,
    GDT_Int32 = 5, GDT_Float32 = 6, GDT_Float64 = 7
} GDALDataType;

inline void* CPLMalloc(size_t n) { return std::malloc(n ? n : 1); }
inline void CPLFree(void* p) { std::free(p); }
inline int GDALGetDataTypeSizeBytes(GDALDataType t) {
    switch (t) {
        case GDT_Byte: return 1;
        case GDT_UInt16: case GDT_Int16: return 2;
        case GDT_Float64: return 8;
        default: return 4;
    }
}
inline char** CSLSetNameValue(char** l, const char*, const char*) { return l; }

class GDALDataset;

class GDALRasterBand {
  public:
    explicit GDALRasterBand(GDALDataset* ds) : ds_(ds) {}
    void GetBlockSize(int* bx, int* by);
    double GetNoDataValue(int* ok = nullptr);
    CPLErr SetNoDataValue(double v);
    CPLErr RasterIO(GDALRWFlag flag, int xoff, int yoff, int xs, int ys, void* buf,
                    int bxs, int bys, GDALDataType t, long, long);
    CPLErr ComputeStatistics(bool, double* mn, double* mx, double* mean, double* sd, void*, void*);
    CPLErr SetStatistics(double, double, double, double) { return CE_None; }
    GDALDataset* ds_;
};

class GDALDataset {
  public:
    mgk_tiff::Raster r;
    std::string path;
    bool writable = false;
    bool dirty = false;
    GDALRasterBand band{this};
    GDALRasterBand* GetRasterBand(int) { return &band; }
    const char* GetProjectionRef() { return r.projection.c_str(); }
    CPLErr GetGeoTransform(double* gt) {
        for (int i = 0; i < 6; i++) gt[i] = r.gt[i];
        return CE_None;
    }
    CPLErr SetGeoTransform(double* gt) {
        for (int i = 0; i < 6; i++) r.gt[i] = gt[i];
        return CE_None;
    }
    CPLErr SetProjection(const char* p) {
        r.projection = p ? p : "";
        return CE_None;
    }
    void FlushCache() {
        if (writable && dirty) {
            if (!mgk_tiff::write_tiff(path, r, 128)) std::fprintf(stderr, "shim: cannot write %s\n", path.c_str());
            dirty = false;
        }
    }
};

inline void GDALRasterBand::GetBlockSize(int* bx, int* by) {
    *bx = ds_->r.block_x > 0 ? ds_->r.block_x : 128;
    *by = ds_->r.block_y > 0 ? ds_->r.block_y : 128;
}
inline double GDALRasterBand::GetNoDataValue(int* ok) {
    if (ok) *ok = ds_->r.has_nodata ? 1 : 0;
    return ds_->r.has_nodata ? ds_->r.nodata : -1e10;
}
inline CPLErr GDALRasterBand::SetNoDataValue(double v) {
    ds_->r.has_nodata = true;
    ds_->r.nodata = v;
    return CE_None;
}
inline CPLErr GDALRasterBand::RasterIO(GDALRWFlag flag, int xoff, int yoff, int xs, int ys, void* buf,
                                       int, int, GDALDataType t, long, long) {
    mgk_tiff::Raster& r = ds_->r;
    if (xoff < 0 || yoff < 0 || xoff + xs > r.ncols || yoff + ys > r.nrows) return CE_Failure;
    for (int y = 0; y < ys; y++)
        for (int x = 0; x < xs; x++) {
            float& cell = r.data[(size_t)(yoff + y) * (size_t)r.ncols + (size_t)(xoff + x)];
            const size_t k = (size_t)y * (size_t)xs + (size_t)x;
            if (flag == GF_Read) {
                if (t == GDT_Float64) ((double*)buf)[k] = cell;
                else ((float*)buf)[k] = cell;
            } else {
                cell = (t == GDT_Float64) ? (float)((double*)buf)[k] : ((float*)buf)[k];
                ds_->dirty = true;
            }
        }
    return CE_None;
}
inline CPLErr GDALRasterBand::ComputeStatistics(bool, double* mn, double* mx, double* mean, double* sd, void*, void*) {
    double a = 1e300, b = -1e300, s = 0, s2 = 0;
    size_t n = 0;
    for (float v : ds_->r.data) {
        if (ds_->r.has_nodata && v == (float)ds_->r.nodata) continue;
        a = std::min(a, (double)v);
        b = std::max(b, (double)v);
        s += v;
        s2 += (double)v * v;
        n++;
    }
    *mn = a; *mx = b;
    *mean = n ? s / n : 0.0;
    *sd = n ? std::sqrt(std::max(0.0, s2 / n - (*mean) * (*mean))) : 0.0;
    return CE_None;
}

class GDALDriver {
  public:
    GDALDataset* Create(const char* name, int ncols, int nrows, int, GDALDataType, char**) {
        GDALDataset* ds = new GDALDataset();
        ds->path = name;
        ds->writable = true;
        ds->dirty = true;
        ds->r.ncols = ncols;
        ds->r.nrows = nrows;
        ds->r.data.assign((size_t)ncols * (size_t)nrows, 0.0f);
        return ds;
    }
};
class GDALDriverManager {
  public:
    GDALDriver* GetDriverByName(const char*) { return &drv_; }
    GDALDriver drv_;
};
inline GDALDriverManager* GetGDALDriverManager() {
    static GDALDriverManager m;
    return &m;
}
inline void GDALAllRegister() {}
inline void GDALDestroyDriverManager() {}
inline GDALDataset* GDALOpen(const char* name, GDALAccess) {
    GDALDataset* ds = new GDALDataset();
    std::string err;
    ds->path = name;
    if (!mgk_tiff::read_tiff(name, ds->r, err)) {
        std::fprintf(stderr, "shim: %s\n", err.c_str());
        std::exit(1);
    }
    return ds;
}
inline void GDALClose(GDALDataset* ds) {
    if (!ds) return;
    ds->FlushCache();
    delete ds;
}
inline int GDALGetRasterXSize(GDALDataset* ds) { return (int)ds->r.ncols; }
inline int GDALGetRasterYSize(GDALDataset* ds) { return (int)ds->r.nrows; }
inline int GDALGetRasterCount(GDALDataset*) { return 1; }
inline GDALDataType GDALGetRasterDataType(GDALRasterBand*) { return GDT_Float32; }
