// Ingest of the measured images (codes_v2/main_run_FPM.m:21-45): one TIFF per LED,
// the pixel region imread(..., 'PixelRegion', {rows, cols}) selects, multi-sample
// pixels averaged as mean(single(temp), 3).  Baseline TIFF only: uncompressed,
// strips, chunky samples of 8 or 16 unsigned bits, either byte order.  Host code:
// it fills a host stack for fpm_solve / fpm_normalise_stack.
#include "tiff.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

namespace fpm {

namespace {

struct File {
    std::FILE *f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

struct Reader {
    std::FILE *f = nullptr;
    bool big = false;  // "MM" byte order
    bool read(uint64_t off, void *dst, size_t n) const {
        return fseeko(f, (off_t)off, SEEK_SET) == 0 && std::fread(dst, 1, n, f) == n;
    }
    uint16_t u16(const uint8_t *p) const {
        return big ? (uint16_t)(p[0] << 8 | p[1]) : (uint16_t)(p[1] << 8 | p[0]);
    }
    uint32_t u32(const uint8_t *p) const {
        return big ? (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]
                   : (uint32_t)p[3] << 24 | (uint32_t)p[2] << 16 | (uint32_t)p[1] << 8 | p[0];
    }
};

struct Entry {
    uint16_t tag = 0, type = 0;
    uint32_t count = 0;
    uint8_t raw[4] = {};
};

// Values of a SHORT (3) or LONG (4) field, inline when they fit in 4 bytes.
bool values(const Reader &rd, const Entry &e, std::vector<uint32_t> &out) {
    const size_t sz = e.type == 3 ? 2 : e.type == 4 ? 4 : 0;
    if (!sz || e.count == 0 || e.count > (1u << 24)) return false;
    std::vector<uint8_t> buf(sz * e.count);
    if (sz * e.count <= 4) {
        std::memcpy(buf.data(), e.raw, sz * e.count);
    } else if (!rd.read(rd.u32(e.raw), buf.data(), buf.size())) {
        return false;
    }
    out.resize(e.count);
    for (uint32_t i = 0; i < e.count; ++i)
        out[i] = sz == 2 ? rd.u16(&buf[2 * i]) : rd.u32(&buf[4 * i]);
    return true;
}

// Layout of the first image of a file (the one imread reads by default).
struct Layout {
    uint32_t width = 0, height = 0, spp = 1, bytes = 0, rows_per_strip = 0;
    std::vector<uint32_t> offsets, counts;
};

std::string parse(Reader &rd, const char *path, Layout &lay) {
    const std::string p(path);
    uint8_t hdr[8];
    if (!rd.read(0, hdr, 8)) return p + ": not a TIFF file";
    if (hdr[0] == 'I' && hdr[1] == 'I') {
        rd.big = false;
    } else if (hdr[0] == 'M' && hdr[1] == 'M') {
        rd.big = true;
    } else {
        return p + ": not a TIFF file";
    }
    const uint16_t magic = rd.u16(hdr + 2);
    if (magic == 43) return p + ": BigTIFF is not supported";
    if (magic != 42) return p + ": not a TIFF file";
    const uint32_t ifd = rd.u32(hdr + 4);
    uint8_t cnt[2];
    if (!rd.read(ifd, cnt, 2)) return p + ": truncated directory";
    const uint16_t n = rd.u16(cnt);
    std::vector<uint8_t> ent(12 * (size_t)n);
    if (!rd.read((uint64_t)ifd + 2, ent.data(), ent.size())) return p + ": truncated directory";
    uint32_t compression = 1, planar = 1, format = 1;
    std::vector<uint32_t> bits;
    for (uint16_t i = 0; i < n; ++i) {
        Entry e;
        const uint8_t *q = &ent[12 * (size_t)i];
        e.tag = rd.u16(q);
        e.type = rd.u16(q + 2);
        e.count = rd.u32(q + 4);
        std::memcpy(e.raw, q + 8, 4);
        std::vector<uint32_t> v;
        switch (e.tag) {
            case 256: if (values(rd, e, v)) lay.width = v[0]; break;
            case 257: if (values(rd, e, v)) lay.height = v[0]; break;
            case 258: values(rd, e, bits); break;
            case 259: if (values(rd, e, v)) compression = v[0]; break;
            case 273: values(rd, e, lay.offsets); break;
            case 277: if (values(rd, e, v)) lay.spp = v[0]; break;
            case 278: if (values(rd, e, v)) lay.rows_per_strip = v[0]; break;
            case 279: values(rd, e, lay.counts); break;
            case 284: if (values(rd, e, v)) planar = v[0]; break;
            case 322: case 323: case 324: case 325:
                return p + ": tiled TIFF is not supported";
            case 339: if (values(rd, e, v)) format = v[0]; break;
            default: break;
        }
    }
    if (lay.width == 0 || lay.height == 0) return p + ": missing image size";
    if (compression != 1) return p + ": compressed TIFF is not supported";
    if (planar != 1 && lay.spp > 1) return p + ": planar samples are not supported";
    if (format != 1) return p + ": samples are not unsigned integers";
    if (lay.spp < 1 || lay.spp > 4) return p + ": unsupported samples per pixel";
    // BitsPerSample defaults to 1 when absent (bilevel), which is not supported
    if (bits.empty()) return p + ": only 8- and 16-bit samples are supported";
    for (uint32_t x : bits)
        if (x != bits[0]) return p + ": mixed sample sizes";
    if (bits[0] != 8 && bits[0] != 16) return p + ": only 8- and 16-bit samples are supported";
    lay.bytes = bits[0] / 8;
    if (lay.rows_per_strip == 0 || lay.rows_per_strip > lay.height) lay.rows_per_strip = lay.height;
    const size_t strips = (lay.height + lay.rows_per_strip - 1) / lay.rows_per_strip;
    if (lay.offsets.size() < strips || lay.counts.size() < strips) return p + ": bad strip table";
    return std::string();
}

void put_rows(const Reader &rd, const Layout &lay, const uint8_t *src, size_t stride, int rows,
              int h, int row_out, TiffOut type, void *page) {
    const uint32_t spp = lay.spp;
    const size_t px = spp * lay.bytes;
    auto sample = [&](const uint8_t *q) -> uint32_t {
        return lay.bytes == 1 ? q[0] : rd.u16(q);
    };
    if (type == TiffOut::kU16) {
        uint16_t *out = static_cast<uint16_t *>(page);
        for (int c = 0; c < h; ++c) {
            uint16_t *dst = out + (size_t)c * h + row_out;
            for (int r = 0; r < rows; ++r) dst[r] = (uint16_t)sample(src + r * stride + c * px);
        }
    } else {
        float *out = static_cast<float *>(page);
        for (int c = 0; c < h; ++c) {
            float *dst = out + (size_t)c * h + row_out;
            for (int r = 0; r < rows; ++r) {
                const uint8_t *q = src + r * stride + c * px;
                // summed in single precision: exact for <= 4 samples of <= 16 bits,
                // then one rounding in the division, as mean(single(x), 3)
                float s = 0.f;
                for (uint32_t k = 0; k < spp; ++k) s += (float)sample(q + k * lay.bytes);
                dst[r] = s / (float)spp;
            }
        }
    }
}

}  // namespace

std::string read_tiff_region(const char *path, int r0, int c0, int h, TiffOut type, void *page) {
    if (!path || !page || h <= 0) return "read_tiff_region: bad arguments";
    File file;
    file.f = std::fopen(path, "rb");
    if (!file.f) return std::string("cannot open ") + path;
    Reader rd;
    rd.f = file.f;
    Layout lay;
    std::string err = parse(rd, path, lay);
    if (!err.empty()) return err;
    const std::string p(path);
    if (type == TiffOut::kU16 && lay.spp != 1)
        return p + ": " + std::to_string(lay.spp) + " samples per pixel need a float stack";
    if (r0 < 0 || c0 < 0 || (uint64_t)r0 + h > lay.height || (uint64_t)c0 + h > lay.width)
        return p + ": pixel region outside the " + std::to_string(lay.height) + " x " +
               std::to_string(lay.width) + " image";
    const size_t px = (size_t)lay.spp * lay.bytes;
    const size_t row_bytes = (size_t)lay.width * px;
    const size_t region_bytes = (size_t)h * px;
    // whole rows in one read when the region covers most of each row
    const bool whole = 2 * region_bytes >= row_bytes;
    constexpr int kPiece = 64;  // rows per read: bounds the buffer, keeps the transpose in cache
    std::vector<uint8_t> buf((size_t)kPiece * (whole ? row_bytes : region_bytes));
    int r = 0;
    while (r < h) {
        const uint32_t y = (uint32_t)(r0 + r);
        const uint32_t s = y / lay.rows_per_strip;
        const uint32_t strip_end = std::min(lay.height, (s + 1) * lay.rows_per_strip);
        const int rows = (int)std::min<uint32_t>({(uint32_t)kPiece, strip_end - y, (uint32_t)(h - r)});
        const uint64_t within = (uint64_t)(y - s * lay.rows_per_strip) * row_bytes;
        if (within + (uint64_t)rows * row_bytes > lay.counts[s])
            return p + ": strip " + std::to_string(s) + " is shorter than its rows";
        size_t stride;
        const uint8_t *src;
        if (whole) {
            if (!rd.read((uint64_t)lay.offsets[s] + within, buf.data(), (size_t)rows * row_bytes))
                return p + ": truncated pixel data";
            stride = row_bytes;
            src = buf.data() + (size_t)c0 * px;
        } else {
            for (int k = 0; k < rows; ++k)
                if (!rd.read((uint64_t)lay.offsets[s] + within + (uint64_t)k * row_bytes + c0 * px,
                             buf.data() + (size_t)k * region_bytes, region_bytes))
                    return p + ": truncated pixel data";
            stride = region_bytes;
            src = buf.data();
        }
        put_rows(rd, lay, src, stride, rows, h, r, type, page);
        r += rows;
    }
    return std::string();
}

std::string read_tiff_stack(const char *const *paths, int n, int r0, int c0, int h, TiffOut type,
                            void *stack, int threads) {
    if (!paths || !stack || n <= 0 || h <= 0) return "read_tiff_stack: bad arguments";
    const size_t page_bytes = (size_t)h * h * (type == TiffOut::kU16 ? 2 : 4);
    if (threads <= 0) threads = (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency()));
    threads = std::min(threads, n);
    std::vector<std::string> errs(n);
    std::atomic<int> next{0};
    auto work = [&] {
        for (int i = next++; i < n; i = next++) {
            errs[i] = paths[i] ? read_tiff_region(paths[i], r0, c0, h, type,
                                                  static_cast<uint8_t *>(stack) + i * page_bytes)
                               : "file name " + std::to_string(i) + " is NULL";
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    for (int i = 0; i < n; ++i)
        if (!errs[i].empty()) return errs[i];
    return std::string();
}

}  // namespace fpm
