// Minimal GeoTIFF reader/writer for single-band rasters (no GDAL).
//
// The reference reads its masks and writes its density surface through GDAL
// (GeoTIFF.cpp:20-577): the reader returns any band type as float, row 0 at
// the top, with the geotransform and NoData value; the writer emits a Float32
// raster tile by tile (GeoTIFF.cpp:552-575).  This header covers the same
// layout without GDAL:
//   read : classic TIFF and BigTIFF, little/big endian, strips or tiles,
//          compression none (1) or LZW (5) with predictor 1/2,
//          8/16/32-bit integer and 32/64-bit float samples -> float
//   write: Float32, uncompressed, tiled, BigTIFF above 4 GiB, with
//          ModelPixelScale/ModelTiepoint and GDAL_NODATA tags, and a
//          region writer so an out-of-core tile loop can stream its tiles.
// Header-only C++17; used by the host driver and by the oracle's build of
// the reference program.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace mgk_tiff {

struct Raster {
    int64_t ncols = 0, nrows = 0;
    double gt[6] = {0, 1, 0, 0, 0, -1};  // GDAL geotransform
    bool has_nodata = false;
    double nodata = 0.0;
    int block_x = 0, block_y = 0;        // tile or strip layout of the file
    std::string projection;              // kept verbatim when present (GeoAsciiParams)
    std::vector<float> data;             // row-major, row 0 = top
};

namespace detail {

struct Reader {
    FILE* f = nullptr;
    bool big_endian = false;
    bool bigtiff = false;
    bool ok = true;

    uint64_t swap(uint64_t v, int n) const {
        if (!big_endian) return v;
        uint64_t r = 0;
        for (int i = 0; i < n; i++) r = (r << 8) | ((v >> (8 * i)) & 0xff);
        return r;
    }
    uint64_t rd(uint64_t off, int n) {
        uint64_t v = 0;
        if (fseeko(f, (off_t)off, SEEK_SET) != 0 || fread(&v, 1, (size_t)n, f) != (size_t)n) {
            ok = false;
            return 0;
        }
        return swap(v, n);
    }
};

inline int type_size(int t) {
    switch (t) {
        case 1: case 2: case 6: case 7: return 1;
        case 3: case 8: return 2;
        case 4: case 9: case 11: return 4;
        case 5: case 10: case 12: case 16: case 17: case 18: return 8;
        default: return 1;
    }
}

struct Entry {
    uint16_t tag = 0, type = 0;
    uint64_t count = 0, value_off = 0;  // offset of the value bytes
};

// LZW decoder for TIFF (MSB-first codes, early change).
inline bool lzw_decode(const uint8_t* in, size_t n, std::vector<uint8_t>& out, size_t expect) {
    out.clear();
    out.reserve(expect);
    std::vector<std::vector<uint8_t>> dict;
    auto reset = [&]() {
        dict.assign(258, {});
        for (int i = 0; i < 256; i++) dict[i] = {(uint8_t)i};
    };
    reset();
    int width = 9;
    uint64_t bitbuf = 0;
    int bits = 0;
    size_t pos = 0;
    int prev = -1;
    while (true) {
        while (bits < width && pos < n) {
            bitbuf = (bitbuf << 8) | in[pos++];
            bits += 8;
        }
        if (bits < width) break;
        int code = (int)((bitbuf >> (bits - width)) & ((1u << width) - 1));
        bits -= width;
        if (code == 257) break;  // EOI
        if (code == 256) {       // clear
            reset();
            width = 9;
            prev = -1;
            continue;
        }
        std::vector<uint8_t> entry;
        if (code < (int)dict.size()) {
            entry = dict[code];
            if (prev >= 0) {
                std::vector<uint8_t> ne = dict[prev];
                ne.push_back(entry[0]);
                dict.push_back(std::move(ne));
            }
        } else if (prev >= 0 && code == (int)dict.size()) {
            entry = dict[prev];
            entry.push_back(dict[prev][0]);
            dict.push_back(entry);
        } else {
            return false;
        }
        out.insert(out.end(), entry.begin(), entry.end());
        prev = code;
        if ((int)dict.size() + 1 >= (1 << width) && width < 12) width++;
    }
    return true;
}

}  // namespace detail

// Reads band 1 of a TIFF into `r`.  Returns false and fills `err` on failure.
inline bool read_tiff(const std::string& path, Raster& r, std::string& err) {
    using namespace detail;
    Reader R;
    R.f = fopen(path.c_str(), "rb");
    if (!R.f) {
        err = "cannot open " + path;
        return false;
    }
    struct Closer { FILE* f; ~Closer() { if (f) fclose(f); } } closer{R.f};
    char hdr[2];
    if (fread(hdr, 1, 2, R.f) != 2) { err = "short file"; return false; }
    if (hdr[0] == 'I' && hdr[1] == 'I') R.big_endian = false;
    else if (hdr[0] == 'M' && hdr[1] == 'M') R.big_endian = true;
    else { err = "not a TIFF"; return false; }
    uint64_t magic = R.rd(2, 2);
    uint64_t ifd;
    if (magic == 42) {
        ifd = R.rd(4, 4);
    } else if (magic == 43) {
        R.bigtiff = true;
        ifd = R.rd(8, 8);
    } else {
        err = "bad TIFF magic";
        return false;
    }
    uint64_t nent = R.rd(ifd, R.bigtiff ? 8 : 2);
    const int esz = R.bigtiff ? 20 : 12;
    const uint64_t base = ifd + (R.bigtiff ? 8 : 2);
    std::vector<Entry> ents;
    for (uint64_t i = 0; i < nent && R.ok; i++) {
        Entry e;
        uint64_t o = base + i * esz;
        e.tag = (uint16_t)R.rd(o, 2);
        e.type = (uint16_t)R.rd(o + 2, 2);
        e.count = R.rd(o + 4, R.bigtiff ? 8 : 4);
        uint64_t vo = o + (R.bigtiff ? 12 : 8);
        uint64_t nbytes = e.count * (uint64_t)type_size(e.type);
        e.value_off = (nbytes <= (uint64_t)(R.bigtiff ? 8 : 4)) ? vo : R.rd(vo, R.bigtiff ? 8 : 4);
        ents.push_back(e);
    }
    if (!R.ok) { err = "truncated IFD"; return false; }
    auto find = [&](int tag) -> const Entry* {
        for (auto& e : ents)
            if (e.tag == tag) return &e;
        return nullptr;
    };
    auto get_uints = [&](int tag) -> std::vector<uint64_t> {
        std::vector<uint64_t> v;
        const Entry* e = find(tag);
        if (!e) return v;
        int ts = type_size(e->type);
        for (uint64_t i = 0; i < e->count; i++) v.push_back(R.rd(e->value_off + i * ts, ts));
        return v;
    };
    auto get_doubles = [&](int tag) -> std::vector<double> {
        std::vector<double> v;
        const Entry* e = find(tag);
        if (!e || e->type != 12) return v;
        for (uint64_t i = 0; i < e->count; i++) {
            uint64_t bits = R.rd(e->value_off + i * 8, 8);
            double d;
            std::memcpy(&d, &bits, 8);
            v.push_back(d);
        }
        return v;
    };
    auto get_ascii = [&](int tag) -> std::string {
        const Entry* e = find(tag);
        if (!e) return std::string();
        std::string s((size_t)e->count, '\0');
        if (fseeko(R.f, (off_t)e->value_off, SEEK_SET) != 0 ||
            fread(&s[0], 1, (size_t)e->count, R.f) != (size_t)e->count)
            return std::string();
        while (!s.empty() && s.back() == '\0') s.pop_back();
        return s;
    };
    auto one = [&](int tag, uint64_t dflt) {
        auto v = get_uints(tag);
        return v.empty() ? dflt : v[0];
    };
    r.ncols = (int64_t)one(256, 0);
    r.nrows = (int64_t)one(257, 0);
    const int bits = (int)one(258, 8);
    const int comp = (int)one(259, 1);
    const int spp = (int)one(277, 1);
    const int fmt = (int)one(339, 1);
    const int pred = (int)one(317, 1);
    const int planar = (int)one(284, 1);
    if (r.ncols <= 0 || r.nrows <= 0) { err = "bad dimensions"; return false; }
    if (comp != 1 && comp != 5) { err = "unsupported compression " + std::to_string(comp); return false; }
    if (pred != 1 && pred != 2) { err = "unsupported predictor"; return false; }
    const int bps = bits / 8;
    const bool tiled = find(322) != nullptr;
    int64_t bw, bh;
    std::vector<uint64_t> offs, cnts;
    if (tiled) {
        bw = (int64_t)one(322, 0);
        bh = (int64_t)one(323, 0);
        offs = get_uints(324);
        cnts = get_uints(325);
    } else {
        bw = r.ncols;
        bh = (int64_t)one(278, (uint64_t)r.nrows);
        if (bh > r.nrows) bh = r.nrows;
        offs = get_uints(273);
        cnts = get_uints(279);
    }
    if (bw <= 0 || bh <= 0 || offs.empty() || offs.size() != cnts.size()) {
        err = "bad block layout";
        return false;
    }
    r.block_x = (int)bw;
    r.block_y = (int)bh;
    const int64_t nbx = (r.ncols + bw - 1) / bw;
    const int64_t nby = (r.nrows + bh - 1) / bh;
    const size_t px_stride = (size_t)(planar == 1 ? spp : 1) * (size_t)bps;
    r.data.assign((size_t)(r.ncols * r.nrows), 0.0f);
    std::vector<uint8_t> raw, dec;
    for (int64_t by = 0; by < nby; by++)
        for (int64_t bx = 0; bx < nbx; bx++) {
            const size_t bi = (size_t)(by * nbx + bx);
            if (bi >= offs.size()) { err = "missing block"; return false; }
            raw.resize((size_t)cnts[bi]);
            if (fseeko(R.f, (off_t)offs[bi], SEEK_SET) != 0 ||
                fread(raw.data(), 1, raw.size(), R.f) != raw.size()) {
                err = "short block read";
                return false;
            }
            const size_t expect = (size_t)bw * (size_t)bh * px_stride;
            const std::vector<uint8_t>* blk = &raw;
            if (comp == 5) {
                if (!lzw_decode(raw.data(), raw.size(), dec, expect)) { err = "bad LZW data"; return false; }
                blk = &dec;
            }
            const int64_t rows_here = std::min<int64_t>(bh, r.nrows - by * bh);
            const int64_t cols_here = std::min<int64_t>(bw, r.ncols - bx * bw);
            for (int64_t yy = 0; yy < rows_here; yy++) {
                const size_t row_off = (size_t)yy * (size_t)bw * px_stride;
                if (row_off + (size_t)cols_here * px_stride > blk->size()) { err = "short block"; return false; }
                const uint8_t* src = blk->data() + row_off;
                std::vector<uint8_t> rowbuf;
                if (pred == 2) {  // horizontal differencing on integer samples
                    rowbuf.assign(src, src + (size_t)bw * px_stride);
                    for (int64_t xx = 1; xx < bw; xx++)
                        for (int b = 0; b < bps; b++) {
                            if (bps == 1) rowbuf[xx] = (uint8_t)(rowbuf[xx] + rowbuf[xx - 1]);
                        }
                    if (bps == 2) {
                        for (int64_t xx = 1; xx < bw; xx++) {
                            uint16_t a, p;
                            std::memcpy(&a, &rowbuf[xx * 2], 2);
                            std::memcpy(&p, &rowbuf[(xx - 1) * 2], 2);
                            a = (uint16_t)(a + p);
                            std::memcpy(&rowbuf[xx * 2], &a, 2);
                        }
                    }
                    src = rowbuf.data();
                }
                float* dst = &r.data[(size_t)((by * bh + yy) * r.ncols + bx * bw)];
                for (int64_t xx = 0; xx < cols_here; xx++) {
                    const uint8_t* s = src + (size_t)xx * px_stride;
                    uint64_t v = 0;
                    std::memcpy(&v, s, (size_t)bps);
                    v = R.swap(v, bps);
                    double val;
                    if (fmt == 3 && bps == 4) { float f; uint32_t u = (uint32_t)v; std::memcpy(&f, &u, 4); val = f; }
                    else if (fmt == 3 && bps == 8) { double d; std::memcpy(&d, &v, 8); val = d; }
                    else if (fmt == 2) { int64_t sv = (int64_t)(v << (64 - 8 * bps)) >> (64 - 8 * bps); val = (double)sv; }
                    else val = (double)v;
                    dst[xx] = (float)val;
                }
            }
        }
    // Georeferencing: ModelPixelScale + ModelTiepoint, or ModelTransformation.
    auto scale = get_doubles(33550);
    auto tie = get_doubles(33922);
    auto mtx = get_doubles(34264);
    if (scale.size() >= 2 && tie.size() >= 6) {
        r.gt[1] = scale[0];
        r.gt[5] = -scale[1];
        r.gt[2] = r.gt[4] = 0.0;
        r.gt[0] = tie[3] - tie[0] * scale[0];
        r.gt[3] = tie[4] + tie[1] * scale[1];
    } else if (mtx.size() >= 8) {
        r.gt[0] = mtx[3]; r.gt[1] = mtx[0]; r.gt[2] = mtx[1];
        r.gt[3] = mtx[7]; r.gt[4] = mtx[4]; r.gt[5] = mtx[5];
    }
    std::string nd = get_ascii(42113);
    if (!nd.empty()) {
        r.has_nodata = true;
        r.nodata = std::strtod(nd.c_str(), nullptr);
    }
    r.projection = get_ascii(34737);
    return true;
}

// Tiled, uncompressed Float32 writer.  The file layout (IFD + tile table)
// is laid down at open; write_region() then stores any rectangle, so tiles
// of a large raster can be written as they are produced.
class TiledWriter {
  public:
    TiledWriter() = default;
    TiledWriter(const TiledWriter&) = delete;
    TiledWriter& operator=(const TiledWriter&) = delete;
    ~TiledWriter() { close(); }

    // resume: reopen an existing file of the same layout (written by an
    // earlier, interrupted run) instead of creating and pre-filling it.
    bool open(const std::string& path, int64_t ncols, int64_t nrows, const double gt[6],
              bool has_nodata, double nodata, int tile = 256, float fill = 0.0f, bool resume = false) {
        close();
        ncols_ = ncols;
        nrows_ = nrows;
        tile_ = tile;
        nbx_ = (ncols + tile - 1) / tile;
        nby_ = (nrows + tile - 1) / tile;
        const uint64_t tile_bytes = (uint64_t)tile * tile * 4;
        const uint64_t data_bytes = tile_bytes * (uint64_t)(nbx_ * nby_);
        big_ = data_bytes > 0xF0000000ull;
        f_ = nullptr;
        // Layout: header | tag payloads | tile offsets | tile counts | IFD | tile data
        std::vector<uint8_t> head;
        auto put = [&](uint64_t v, int n) {
            for (int i = 0; i < n; i++) head.push_back((uint8_t)(v >> (8 * i)));
        };
        const int osz = big_ ? 8 : 4;
        put('I' | ('I' << 8), 2);
        if (big_) { put(43, 2); put(8, 2); put(0, 2); put(0, 8); }  // IFD offset patched below
        else { put(42, 2); put(0, 4); }
        const size_t ifd_ptr_pos = big_ ? 8 : 4;
        const uint64_t ntiles = (uint64_t)(nbx_ * nby_);
        // payloads
        auto align8 = [&]() { while (head.size() % 8) head.push_back(0); };
        align8();
        const uint64_t scale_off = head.size();
        double scale[3] = {gt[1], -gt[5], 0.0};
        for (double d : scale) { uint64_t b; std::memcpy(&b, &d, 8); put(b, 8); }
        const uint64_t tie_off = head.size();
        double tie[6] = {0, 0, 0, gt[0], gt[3], 0};
        for (double d : tie) { uint64_t b; std::memcpy(&b, &d, 8); put(b, 8); }
        char ndbuf[64];
        std::snprintf(ndbuf, sizeof(ndbuf), "%.17g", nodata);
        const std::string nds = std::string(ndbuf);
        const uint64_t nd_off = head.size();
        for (char c : nds) head.push_back((uint8_t)c);
        head.push_back(0);
        align8();
        const uint64_t toff_off = head.size();
        head.resize(head.size() + ntiles * osz, 0);
        const uint64_t tcnt_off = head.size();
        for (uint64_t i = 0; i < ntiles; i++) put(tile_bytes, osz);
        align8();
        // IFD
        struct Tag { uint16_t tag, type; uint64_t count, value; };
        std::vector<Tag> tags = {
            {256, big_ ? (uint16_t)16 : (uint16_t)4, 1, (uint64_t)ncols},
            {257, big_ ? (uint16_t)16 : (uint16_t)4, 1, (uint64_t)nrows},
            {258, 3, 1, 32},
            {259, 3, 1, 1},
            {262, 3, 1, 1},
            {277, 3, 1, 1},
            {284, 3, 1, 1},
            {322, 3, 1, (uint64_t)tile},
            {323, 3, 1, (uint64_t)tile},
            {324, big_ ? (uint16_t)16 : (uint16_t)4, ntiles, ntiles == 1 ? 0 : toff_off},
            {325, big_ ? (uint16_t)16 : (uint16_t)4, ntiles, ntiles == 1 ? tile_bytes : tcnt_off},
            {339, 3, 1, 3},
            {33550, 12, 3, scale_off},
            {33922, 12, 6, tie_off},
        };
        if (has_nodata) tags.push_back({42113, 2, (uint64_t)nds.size() + 1,
                                        nds.size() + 1 <= (size_t)osz ? 0 : nd_off});
        const uint64_t ifd_off = head.size();
        put(tags.size(), big_ ? 8 : 2);
        size_t single_tile_value_pos = 0;
        for (auto& t : tags) {
            put(t.tag, 2);
            put(t.type, 2);
            put(t.count, big_ ? 8 : 4);
            if (t.tag == 324 && ntiles == 1) single_tile_value_pos = head.size();
            if (t.tag == 42113 && nds.size() + 1 <= (size_t)osz) {
                uint64_t v = 0;
                std::memcpy(&v, nds.c_str(), nds.size());
                put(v, osz);
            } else {
                put(t.value, osz);
            }
        }
        put(0, osz);  // next IFD
        align8();
        data_off_ = head.size();
        // patch IFD pointer and tile offsets
        for (int i = 0; i < (big_ ? 8 : 4); i++) head[ifd_ptr_pos + i] = (uint8_t)(ifd_off >> (8 * i));
        if (ntiles == 1) {
            for (int i = 0; i < osz; i++) head[single_tile_value_pos + i] = (uint8_t)(data_off_ >> (8 * i));
        } else {
            for (uint64_t t = 0; t < ntiles; t++) {
                uint64_t o = data_off_ + t * tile_bytes;
                for (int i = 0; i < osz; i++) head[toff_off + t * osz + i] = (uint8_t)(o >> (8 * i));
            }
        }
        const uint64_t total = data_off_ + ntiles * tile_bytes;
        if (resume) {
            f_ = fopen(path.c_str(), "r+b");
            if (f_) {
                std::vector<uint8_t> have(head.size());
                const bool same = fseeko(f_, 0, SEEK_END) == 0 && (uint64_t)ftello(f_) == total &&
                                  fseeko(f_, 0, SEEK_SET) == 0 &&
                                  fread(have.data(), 1, have.size(), f_) == have.size() && have == head;
                if (same) return true;
                fclose(f_);
                f_ = nullptr;
            }
            return false;  // missing, or not the file this run would write
        }
        f_ = fopen(path.c_str(), "w+b");
        if (!f_) return false;
        if (fwrite(head.data(), 1, head.size(), f_) != head.size()) return false;
        // pre-fill tile data
        std::vector<float> fillbuf((size_t)tile * tile, fill);
        for (uint64_t t = 0; t < ntiles; t++)
            if (fwrite(fillbuf.data(), 4, fillbuf.size(), f_) != fillbuf.size()) return false;
        return true;
    }

    // Writes rows [yoff, yoff+ny) x cols [xoff, xoff+nx) from a row-major buffer.
    bool write_region(int64_t xoff, int64_t yoff, int64_t nx, int64_t ny, const float* buf) {
        if (!f_ || xoff < 0 || yoff < 0 || xoff + nx > ncols_ || yoff + ny > nrows_) return false;
        const uint64_t tile_bytes = (uint64_t)tile_ * tile_ * 4;
        for (int64_t y = 0; y < ny; y++) {
            const int64_t gy = yoff + y;
            const int64_t ty = gy / tile_, iy = gy % tile_;
            int64_t x = 0;
            while (x < nx) {
                const int64_t gx = xoff + x;
                const int64_t tx = gx / tile_, ix = gx % tile_;
                const int64_t run = std::min<int64_t>(nx - x, tile_ - ix);
                const uint64_t off = data_off_ + (uint64_t)(ty * nbx_ + tx) * tile_bytes +
                                     ((uint64_t)iy * tile_ + (uint64_t)ix) * 4;
                if (fseeko(f_, (off_t)off, SEEK_SET) != 0) return false;
                if (fwrite(buf + y * nx + x, 4, (size_t)run, f_) != (size_t)run) return false;
                x += run;
            }
        }
        return true;
    }

    bool flush() { return f_ && fflush(f_) == 0; }

    void close() {
        if (f_) fclose(f_);
        f_ = nullptr;
    }

  private:
    FILE* f_ = nullptr;
    bool big_ = false;
    int64_t ncols_ = 0, nrows_ = 0, nbx_ = 0, nby_ = 0;
    int tile_ = 256;
    uint64_t data_off_ = 0;
};

inline bool write_tiff(const std::string& path, const Raster& r, int tile = 256) {
    TiledWriter w;
    if (!w.open(path, r.ncols, r.nrows, r.gt, r.has_nodata, r.nodata, tile)) return false;
    if (!w.write_region(0, 0, r.ncols, r.nrows, r.data.data())) return false;
    w.close();
    return true;
}

}  // namespace mgk_tiff
