// maps.cpp -- SpatiallyExplicit map input: one-band (Geo)TIFF files and the
// reference's map fix-ups.
//
// load: rustcoalescence/scenarios/src/spatially_explicit/maps/tiff/mod.rs:27-127
//   (load_map_from_tiff).  The first image of a baseline TIFF or BigTIFF,
//   little or big endian, in strips or tiles, uncompressed, LZW, PackBits or
//   Deflate, with no, horizontal or floating-point prediction.  Like the
//   reference: the image must be Gray (PhotometricInterpretation 0 or 1) with
//   one sample per pixel of the requested bit width (32 for habitat maps,
//   64 for dispersal and turnover maps); a SampleFormat tag, when present,
//   must be Uint (habitat) or IEEEFP (dispersal, turnover), and an f64 map
//   must be IEEEFP to decode as f64 at all.  Unless loading is strict, a GDAL
//   no-data value (tag 42113, ASCII) parsed as the map's type replaces equal
//   samples by 0.
// fix: maps/mod.rs:11-215 (load_dispersal_map / load_turnover_map
//   non-negativity checks, fix_habitat_map, fix_no_turnover_habitat_map,
//   fix_dispersal_map) under the loading modes FixMe, OffByOne (the
//   reference's default) and Strict.
#include <zlib.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/necsim_b200.h"

namespace {

struct MapError {
    int code;
    std::string msg;
};

[[noreturn]] void bad(const std::string &msg, int code = NECSIM_E_INVALID_ARGUMENT) { throw MapError{code, msg}; }

// ---- file access ----
struct Bytes {
    std::vector<uint8_t> b;
    bool big = false;

    void need(uint64_t off, uint64_t n) const {
        if (off > b.size() || n > b.size() - off) bad("truncated TIFF file (read past its end)");
    }
    uint64_t get(uint64_t off, int size) const {
        need(off, (uint64_t)size);
        uint64_t v = 0;
        for (int j = 0; j < size; ++j) {
            const uint64_t byte = b[off + (uint64_t)j];
            v |= big ? byte << (8 * (size - 1 - j)) : byte << (8 * j);
        }
        return v;
    }
};

// ---- the first image file directory ----
struct Entry {
    uint16_t type = 0;
    uint64_t count = 0;
    uint64_t at = 0;  // file offset of the value(s)
};

int type_size(uint16_t type) {
    switch (type) {
    case 1: case 2: case 6: case 7: return 1;  // BYTE ASCII SBYTE UNDEFINED
    case 3: case 8: return 2;                  // SHORT SSHORT
    case 4: case 9: case 11: case 13: return 4;  // LONG SLONG FLOAT IFD
    case 5: case 10: case 12: case 16: case 17: case 18: return 8;  // RATIONAL DOUBLE LONG8 ...
    default: return 0;
    }
}

struct Ifd {
    const Bytes *f = nullptr;
    std::vector<std::pair<uint16_t, Entry>> entries;

    const Entry *find(uint16_t tag) const {
        for (auto &e : entries)
            if (e.first == tag) return &e.second;
        return nullptr;
    }
    // unsigned integer values (BYTE, SHORT, LONG, LONG8, IFD)
    std::vector<uint64_t> uints(uint16_t tag, const char *name) const {
        const Entry *e = find(tag);
        if (!e) return {};
        const int s = type_size(e->type);
        if (!(e->type == 1 || e->type == 3 || e->type == 4 || e->type == 16 || e->type == 13))
            bad(std::string("TIFF tag ") + name + " does not hold unsigned integers");
        if (e->count > f->b.size()) bad("truncated TIFF file (read past its end)");
        f->need(e->at, e->count * (uint64_t)s);  // before allocating for a corrupt count
        std::vector<uint64_t> v(e->count);
        for (uint64_t j = 0; j < e->count; ++j) v[j] = f->get(e->at + j * (uint64_t)s, s);
        return v;
    }
    uint64_t uint1(uint16_t tag, const char *name, uint64_t dflt, bool required = false) const {
        const std::vector<uint64_t> v = uints(tag, name);
        if (v.empty()) {
            if (required) bad(std::string("required TIFF tag ") + name + " not found");
            return dflt;
        }
        return v[0];
    }
};

// reads the byte order mark into f.big, then the first IFD's entries
Ifd first_ifd(Bytes &f) {
    if (f.b.size() < 8) bad("not a TIFF file (too short)");
    if (f.b[0] == 'I' && f.b[1] == 'I') f.big = false;
    else if (f.b[0] == 'M' && f.b[1] == 'M') f.big = true;
    else bad("not a TIFF file (byte order mark)");
    const uint64_t magic = f.get(2, 2);
    Ifd ifd;
    ifd.f = &f;
    if (magic == 42) {
        const uint64_t off = f.get(4, 4);
        const uint64_t n = f.get(off, 2);
        for (uint64_t j = 0; j < n; ++j) {
            const uint64_t at = off + 2 + 12 * j;
            Entry e;
            const uint16_t tag = (uint16_t)f.get(at, 2);
            e.type = (uint16_t)f.get(at + 2, 2);
            e.count = f.get(at + 4, 4);
            const int s = type_size(e.type);
            if (s == 0) continue;  // unknown types are skipped, like unknown tags
            e.at = (e.count * (uint64_t)s <= 4) ? at + 8 : f.get(at + 8, 4);
            ifd.entries.push_back({tag, e});
        }
    } else if (magic == 43) {  // BigTIFF
        if (f.get(4, 2) != 8) bad("BigTIFF with an offset size other than 8");
        const uint64_t off = f.get(8, 8);
        const uint64_t n = f.get(off, 8);
        for (uint64_t j = 0; j < n; ++j) {
            const uint64_t at = off + 8 + 20 * j;
            Entry e;
            const uint16_t tag = (uint16_t)f.get(at, 2);
            e.type = (uint16_t)f.get(at + 2, 2);
            e.count = f.get(at + 4, 8);
            const int s = type_size(e.type);
            if (s == 0) continue;
            e.at = (e.count * (uint64_t)s <= 8) ? at + 12 : f.get(at + 12, 8);
            ifd.entries.push_back({tag, e});
        }
    } else {
        bad("not a TIFF file (magic number)");
    }
    return ifd;
}

// ---- decompression ----

// TIFF LZW (TIFF 6.0 section 13): MSB-first codes of 9..12 bits, Clear 256,
// EndOfInformation 257, the code width growing one code early
void lzw_decode(const uint8_t *src, size_t n, std::vector<uint8_t> &out, size_t want) {
    constexpr int kClear = 256, kEoi = 257, kMax = 4096;
    std::vector<uint16_t> prefix(kMax);
    std::vector<uint8_t> last(kMax), first(kMax);
    std::vector<uint16_t> len(kMax);
    for (int j = 0; j < 256; ++j) {
        prefix[j] = 0xffff;
        last[j] = first[j] = (uint8_t)j;
        len[j] = 1;
    }
    int next = 258, width = 9, old = -1;
    uint64_t bitpos = 0;
    const uint64_t nbits = (uint64_t)n * 8;
    auto emit = [&](int code) {
        const size_t l = len[code];
        const size_t at = out.size();
        out.resize(at + l);
        for (size_t k = l; k-- > 0;) {
            out[at + k] = last[code];
            code = prefix[code];
        }
    };
    while (out.size() < want) {
        if (bitpos + (uint64_t)width > nbits) break;  // data ended without EOI
        int code = 0;
        for (int k = 0; k < width; ++k, ++bitpos)
            code = (code << 1) | ((src[bitpos >> 3] >> (7 - (bitpos & 7))) & 1);
        if (code == kEoi) break;
        if (code == kClear) {
            next = 258;
            width = 9;
            old = -1;
            continue;
        }
        if (old < 0) {
            if (code > 255) bad("corrupt LZW data (first code after Clear is not a literal)");
            emit(code);
            old = code;
            continue;
        }
        if (code > next || (code == next && next >= kMax)) bad("corrupt LZW data (code out of range)");
        const bool known = code < next;
        const uint8_t head = known ? first[code] : first[old];
        if (next < kMax) {
            prefix[next] = (uint16_t)old;
            last[next] = head;
            first[next] = first[old];
            len[next] = (uint16_t)(len[old] + 1);
            ++next;
        }
        emit(code);
        old = code;
        if (next + 1 >= (1 << width) && width < 12) ++width;
    }
}

void packbits_decode(const uint8_t *src, size_t n, std::vector<uint8_t> &out, size_t want) {
    size_t i = 0;
    while (i < n && out.size() < want) {
        const int8_t h = (int8_t)src[i++];
        if (h >= 0) {
            const size_t k = (size_t)h + 1;
            if (i + k > n) bad("corrupt PackBits data");
            out.insert(out.end(), src + i, src + i + k);
            i += k;
        } else if (h != -128) {
            if (i >= n) bad("corrupt PackBits data");
            out.insert(out.end(), (size_t)(1 - h), src[i++]);
        }
    }
}

void deflate_decode(const uint8_t *src, size_t n, std::vector<uint8_t> &out, size_t want) {
    out.resize(want);
    z_stream z;
    std::memset(&z, 0, sizeof(z));
    if (inflateInit(&z) != Z_OK) bad("zlib initialisation failed");
    z.next_in = const_cast<Bytef *>(src);
    z.avail_in = (uInt)n;
    z.next_out = out.data();
    z.avail_out = (uInt)want;
    const int rc = inflate(&z, Z_FINISH);
    const size_t got = want - z.avail_out;
    inflateEnd(&z);
    if (rc != Z_STREAM_END && rc != Z_BUF_ERROR && rc != Z_OK) bad("corrupt Deflate data");
    out.resize(got);
}

// one strip or tile, decompressed to exactly `want` bytes
std::vector<uint8_t> decompress(uint64_t compression, const uint8_t *src, size_t n, size_t want) {
    std::vector<uint8_t> out;
    out.reserve(want);
    switch (compression) {
    case 1: out.assign(src, src + std::min(n, want)); break;
    case 5: lzw_decode(src, n, out, want); break;
    case 8: case 32946: deflate_decode(src, n, out, want); break;
    case 32773: packbits_decode(src, n, out, want); break;
    default: bad("unsupported TIFF compression " + std::to_string(compression));
    }
    if (out.size() < want) bad("TIFF strip or tile holds fewer samples than its size");
    out.resize(want);
    return out;
}

// ---- samples ----
uint64_t load_sample(const uint8_t *p, int bytes, bool big) {
    uint64_t v = 0;
    for (int j = 0; j < bytes; ++j) v |= (uint64_t)p[j] << (8 * (big ? bytes - 1 - j : j));
    return v;
}
void store_sample(uint8_t *p, int bytes, uint64_t v) {  // host (little endian) order
    for (int j = 0; j < bytes; ++j) p[j] = (uint8_t)(v >> (8 * j));
}

// undoes the predictor over one block of `rows` x `cols` samples and turns
// them into host byte order
void unpredict(std::vector<uint8_t> &blk, uint64_t rows, uint64_t cols, int bytes, bool big, uint64_t predictor) {
    const uint64_t rb = cols * (uint64_t)bytes;
    const uint64_t mask = bytes == 8 ? ~0ULL : ((1ULL << (8 * bytes)) - 1);
    for (uint64_t r = 0; r < rows; ++r) {
        uint8_t *row = blk.data() + r * rb;
        if (predictor == 3) {
            // floating-point predictor: bytes differenced along the row, the
            // row stored as all samples' most significant bytes first
            for (uint64_t j = 1; j < rb; ++j) row[j] = (uint8_t)(row[j] + row[j - 1]);
            std::vector<uint8_t> tmp(row, row + rb);
            for (uint64_t c = 0; c < cols; ++c) {
                uint64_t v = 0;
                for (int k = 0; k < bytes; ++k) v = (v << 8) | tmp[(uint64_t)k * cols + c];
                store_sample(row + c * (uint64_t)bytes, bytes, v);
            }
            continue;
        }
        uint64_t prev = 0;
        for (uint64_t c = 0; c < cols; ++c) {
            uint64_t v = load_sample(row + c * (uint64_t)bytes, bytes, big);
            if (predictor == 2 && c > 0) v = (v + prev) & mask;  // horizontal differencing
            store_sample(row + c * (uint64_t)bytes, bytes, v);
            prev = v;
        }
    }
}

struct Image {
    uint32_t width = 0, height = 0;
    std::vector<uint8_t> data;  // host-order samples, row-major
};

// load_map_from_tiff (maps/tiff/mod.rs:27-127) up to the no-data handling
Image read_tiff(const char *path, int bits, uint64_t want_format, std::string *nodata) {
    Bytes f;
    {
        FILE *fp = std::fopen(path, "rb");
        if (!fp) bad(std::string("could not read file ") + path + ": " + std::strerror(errno));
        std::fseek(fp, 0, SEEK_END);
        const long size = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        f.b.resize(size > 0 ? (size_t)size : 0);
        const size_t got = f.b.empty() ? 0 : std::fread(f.b.data(), 1, f.b.size(), fp);
        std::fclose(fp);
        if (got != f.b.size()) bad(std::string("could not read file ") + path);
    }
    const Ifd ifd = first_ifd(f);
    Image im;
    const uint64_t w = ifd.uint1(256, "ImageWidth", 0, true);
    const uint64_t h = ifd.uint1(257, "ImageLength", 0, true);
    if (w == 0 || h == 0 || w > 0xffffffffULL || h > 0xffffffffULL) bad("TIFF image dimensions out of range");
    if (w > (1ULL << 40) / h) bad("TIFF image too large");  // keeps w * h * 8 far from overflow
    const uint64_t spp = ifd.uint1(277, "SamplesPerPixel", 1);
    const uint64_t photometric = ifd.uint1(262, "PhotometricInterpretation", 0, true);
    std::vector<uint64_t> bps = ifd.uints(258, "BitsPerSample");
    if (bps.empty()) bps.assign(1, 1);
    if (spp != 1) bad("Image must only have one sample per pixel but has " + std::to_string(spp) + ".");
    if (photometric > 1) bad("Image data format is not Gray (one band)");
    if (bps[0] != (uint64_t)bits)
        bad("Image data format Gray(" + std::to_string(bps[0]) + ") does not use the correct bitwidth " +
            std::to_string(bits) + ".");
    const std::vector<uint64_t> fmt = ifd.uints(339, "SampleFormat");
    if (!fmt.empty() && fmt[0] != want_format)
        bad("Image data must have the sample format " + std::string(want_format == 3 ? "IEEEFP" : "Uint") +
            " but has " + std::to_string(fmt[0]) + ".");
    if (fmt.empty() && want_format != 1) bad("Failed to decode the image data as f64 (no IEEEFP SampleFormat).");
    const uint64_t compression = ifd.uint1(259, "Compression", 1);
    const uint64_t predictor = ifd.uint1(317, "Predictor", 1);
    if (predictor < 1 || predictor > 3) bad("unsupported TIFF predictor " + std::to_string(predictor));
    if (predictor == 3 && want_format != 3) bad("floating-point predictor on integer samples");
    const int bytes = bits / 8;
    im.width = (uint32_t)w;
    im.height = (uint32_t)h;
    im.data.assign(w * h * (uint64_t)bytes, 0);

    const bool tiled = ifd.find(322) != nullptr;
    if (!tiled) {
        const uint64_t rps = std::min<uint64_t>(ifd.uint1(278, "RowsPerStrip", 0xffffffffULL), h);
        const std::vector<uint64_t> offs = ifd.uints(273, "StripOffsets");
        const std::vector<uint64_t> lens = ifd.uints(279, "StripByteCounts");
        const uint64_t strips = (h + rps - 1) / rps;
        if (rps == 0 || offs.size() < strips || lens.size() < strips) bad("TIFF strip tags are inconsistent");
        for (uint64_t s = 0; s < strips; ++s) {
            const uint64_t rows = std::min(rps, h - s * rps);
            f.need(offs[s], lens[s]);
            std::vector<uint8_t> blk =
                decompress(compression, f.b.data() + offs[s], (size_t)lens[s], (size_t)(rows * w * (uint64_t)bytes));
            unpredict(blk, rows, w, bytes, f.big, predictor);
            std::memcpy(im.data.data() + s * rps * w * (uint64_t)bytes, blk.data(), blk.size());
        }
    } else {
        const uint64_t tw = ifd.uint1(322, "TileWidth", 0, true);
        const uint64_t th = ifd.uint1(323, "TileLength", 0, true);
        const std::vector<uint64_t> offs = ifd.uints(324, "TileOffsets");
        const std::vector<uint64_t> lens = ifd.uints(325, "TileByteCounts");
        if (tw == 0 || th == 0) bad("TIFF tile size is zero");
        const uint64_t across = (w + tw - 1) / tw, down = (h + th - 1) / th;
        if (offs.size() < across * down || lens.size() < across * down) bad("TIFF tile tags are inconsistent");
        for (uint64_t ty = 0; ty < down; ++ty)
            for (uint64_t tx = 0; tx < across; ++tx) {
                const uint64_t t = ty * across + tx;
                f.need(offs[t], lens[t]);
                std::vector<uint8_t> blk =
                    decompress(compression, f.b.data() + offs[t], (size_t)lens[t], (size_t)(tw * th * (uint64_t)bytes));
                unpredict(blk, th, tw, bytes, f.big, predictor);
                const uint64_t rows = std::min(th, h - ty * th), cols = std::min(tw, w - tx * tw);
                for (uint64_t r = 0; r < rows; ++r)
                    std::memcpy(im.data.data() + ((ty * th + r) * w + tx * tw) * (uint64_t)bytes,
                                blk.data() + r * tw * (uint64_t)bytes, cols * (uint64_t)bytes);
            }
    }
    if (nodata) {
        nodata->clear();
        if (const Entry *e = ifd.find(42113)) {
            if (e->type != 2) bad("GDAL nodata tag is not ASCII");
            f.need(e->at, e->count);
            for (uint64_t j = 0; j < e->count && f.b[e->at + j] != 0; ++j) nodata->push_back((char)f.b[e->at + j]);
            if (nodata->empty()) nodata->push_back('\0');  // present but empty: fails to parse below
        }
    }
    return im;
}

// Rust's `str::parse::<u32>` (decimal digits, optional leading '+')
bool parse_u32(const std::string &s, uint32_t &v) {
    size_t i = (!s.empty() && s[0] == '+') ? 1 : 0;
    if (i >= s.size()) return false;
    uint64_t x = 0;
    for (; i < s.size(); ++i) {
        if (s[i] < '0' || s[i] > '9') return false;
        x = x * 10 + (uint64_t)(s[i] - '0');
        if (x > 0xffffffffULL) return false;
    }
    v = (uint32_t)x;
    return true;
}

// Rust's `str::parse::<f64>`: an optional sign, then inf / infinity / nan
// (any case) or a decimal number with optional exponent; no whitespace
bool parse_f64(const std::string &s, double &v) {
    if (s.empty()) return false;
    size_t i = (s[0] == '+' || s[0] == '-') ? 1 : 0;
    std::string rest = s.substr(i);
    std::string low;
    for (char c : rest) low.push_back((char)std::tolower((unsigned char)c));
    const bool neg = s[0] == '-';
    if (low == "inf" || low == "infinity") {
        v = neg ? -INFINITY : INFINITY;
        return true;
    }
    if (low == "nan") {
        v = NAN;
        return true;
    }
    bool digits = false, dot = false;
    size_t k = 0;
    for (; k < rest.size(); ++k) {
        const char c = rest[k];
        if (c >= '0' && c <= '9') digits = true;
        else if (c == '.' && !dot) dot = true;
        else break;
    }
    if (!digits) return false;
    if (k < rest.size()) {
        if (rest[k] != 'e' && rest[k] != 'E') return false;
        size_t e = k + 1;
        if (e < rest.size() && (rest[e] == '+' || rest[e] == '-')) ++e;
        if (e >= rest.size()) return false;
        for (; e < rest.size(); ++e)
            if (rest[e] < '0' || rest[e] > '9') return false;
    }
    errno = 0;
    char *end = nullptr;
    v = std::strtod(s.c_str(), &end);  // correctly rounded, as Rust's parser is
    return end == s.c_str() + s.size();
}

int fill_err(char *buf, size_t cap, const std::string &msg) {
    if (buf && cap) {
        std::snprintf(buf, cap, "%s", msg.c_str());
    }
    return 0;
}

}  // namespace

extern "C" {

int necsim_map_load(const char *path, int32_t sample, int32_t strict, void **data, uint32_t *width,
                    uint32_t *height, char *err, size_t err_cap) {
    if (!path || !data || !width || !height || (sample != NECSIM_MAP_U32 && sample != NECSIM_MAP_F64)) {
        fill_err(err, err_cap, "invalid argument");
        return NECSIM_E_INVALID_ARGUMENT;
    }
    *data = nullptr;
    try {
        std::string nodata;
        const bool f64 = sample == NECSIM_MAP_F64;
        Image im = read_tiff(path, f64 ? 64 : 32, f64 ? 3 : 1, strict ? nullptr : &nodata);
        const uint64_t n = (uint64_t)im.width * im.height;
        if (!strict && !nodata.empty()) {
            if (f64) {
                double nd;
                if (!parse_f64(nodata, nd)) bad("Could not interpret GDAL nodata value \"" + nodata + "\" as f64.");
                double *p = reinterpret_cast<double *>(im.data.data());
                for (uint64_t j = 0; j < n; ++j)
                    if (p[j] == nd) p[j] = 0.0;
            } else {
                uint32_t nd;
                if (!parse_u32(nodata, nd)) bad("Could not interpret GDAL nodata value \"" + nodata + "\" as u32.");
                uint32_t *p = reinterpret_cast<uint32_t *>(im.data.data());
                for (uint64_t j = 0; j < n; ++j)
                    if (p[j] == nd) p[j] = 0;
            }
        }
        void *out = std::malloc(im.data.size());
        if (!out) bad("out of host memory", NECSIM_E_OUT_OF_MEMORY);
        std::memcpy(out, im.data.data(), im.data.size());
        *data = out;
        *width = im.width;
        *height = im.height;
        fill_err(err, err_cap, "");
        return NECSIM_OK;
    } catch (const MapError &e) {
        fill_err(err, err_cap, std::string(path) + ": " + e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        fill_err(err, err_cap, "out of host memory");
        return NECSIM_E_OUT_OF_MEMORY;
    }
}

void necsim_map_free(void *data) { std::free(data); }

int necsim_maps_fix(uint32_t *habitat, uint32_t width, uint32_t height, double *dispersal, uint64_t dispersal_rows,
                    uint64_t dispersal_cols, const double *turnover, int32_t mode, char *err, size_t err_cap) {
    const uint64_t w = width, h = height, size = w * h;
    if (!habitat || !dispersal || size == 0 || mode < NECSIM_MAPS_OFF_BY_ONE || mode > NECSIM_MAPS_STRICT) {
        fill_err(err, err_cap, "invalid argument");
        return NECSIM_E_INVALID_ARGUMENT;
    }
    // load_dispersal_map / load_turnover_map (maps/mod.rs:11-53)
    for (uint64_t j = 0; j < dispersal_rows * dispersal_cols; ++j)
        if (dispersal[j] < 0.0) {
            fill_err(err, err_cap, "Dispersal weights are not all non-negative");
            return NECSIM_E_DISPERSAL_MAP;
        }
    if (turnover)
        for (uint64_t j = 0; j < size; ++j)
            if (turnover[j] < 0.0) {
                fill_err(err, err_cap, "Turnover rates are not all non-negative");
                return NECSIM_E_INVALID_ARGUMENT;
            }
    if (mode == NECSIM_MAPS_STRICT) return NECSIM_OK;
    // fix_habitat_map (maps/mod.rs:90-130): habitat 0/1 follows turnover and
    // whether any dispersal leaves the cell
    for (uint64_t y = 0; y < h; ++y)
        for (uint64_t x = 0; x < w; ++x) {
            const uint64_t cell = y * w + x;
            if (habitat[cell] > 1) continue;
            uint32_t fixed = 0;
            if (turnover && turnover[cell] == 0.0) {
                fixed = 0;
            } else if (cell < dispersal_rows) {
                const double *row = dispersal + cell * dispersal_cols;
                for (uint64_t c = 0; c < dispersal_cols; ++c)
                    if (row[c] > 0.0) {
                        fixed = 1;
                        break;
                    }
            }
            habitat[cell] = fixed;
        }
    if (mode == NECSIM_MAPS_OFF_BY_ONE) return NECSIM_OK;
    // fix_no_turnover_habitat_map (maps/mod.rs:133-154)
    if (turnover)
        for (uint64_t j = 0; j < size; ++j)
            if (turnover[j] == 0.0) habitat[j] = 0;
    // fix_dispersal_map (maps/mod.rs:158-215), which indexes the map as
    // (w*h) x (w*h)
    if (dispersal_rows != size || dispersal_cols != size) {
        fill_err(err, err_cap, "the dispersal map is not (width*height) x (width*height)");
        return NECSIM_E_DISPERSAL_MAP;
    }
    for (uint64_t row = 0; row < size; ++row) {
        double *d = dispersal + row * size;
        if (habitat[row] == 0) {
            for (uint64_t c = 0; c < size; ++c)
                if (d[c] > 0.0) d[c] = 0.0;
        } else {
            double total = 0.0;
            for (uint64_t c = 0; c < size; ++c) {
                if (habitat[c] == 0 && d[c] > 0.0) d[c] = 0.0;
                total += d[c];
            }
            if (total <= 0.0) d[row] = 1.0;
        }
    }
    return NECSIM_OK;
}

}  // extern "C"
