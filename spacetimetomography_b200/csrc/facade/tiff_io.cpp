// tiff_io.cpp -- the file formats the reference reads and writes through CImg
// (S/ImageFormationModel/CImg.h, built there with libtiff): uncompressed
// baseline TIFF stacks (the projection stack, S/ST_Tomo/ST_Tomography.cpp:355;
// the initial volumes, S/ImageFormationModel/VolumeData.cpp:119; every SART
// output, ST_Tomography.cpp:805) and the Analyze 7.5 flow field
// (ST_Tomography.cpp:467).  Written from the TIFF 6.0 and Analyze 7.5 layouts.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "stt_host.h"

namespace stt_facade {
void set_error(const std::string &m);
}

namespace {

using stt_facade::set_error;

struct Reader {
    std::vector<unsigned char> buf;
    bool be = false;  // big-endian file
    bool ok(size_t off, size_t n) const { return off <= buf.size() && n <= buf.size() - off; }
    uint16_t u16(size_t o) const {
        return be ? (uint16_t)((buf[o] << 8) | buf[o + 1]) : (uint16_t)(buf[o] | (buf[o + 1] << 8));
    }
    uint32_t u32(size_t o) const {
        return be ? ((uint32_t)buf[o] << 24) | ((uint32_t)buf[o + 1] << 16) | ((uint32_t)buf[o + 2] << 8) | buf[o + 3]
                  : (uint32_t)buf[o] | ((uint32_t)buf[o + 1] << 8) | ((uint32_t)buf[o + 2] << 16) |
                        ((uint32_t)buf[o + 3] << 24);
    }
    uint64_t u64(size_t o) const {
        uint64_t a = u32(o), b = u32(o + 4);
        return be ? (a << 32) | b : (b << 32) | a;
    }
};

bool read_file(const char *path, std::vector<unsigned char> &out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        set_error(std::string("cannot open ") + path + ": " + std::strerror(errno));
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(n > 0 ? (size_t)n : 0);
    const bool good = n <= 0 || std::fread(out.data(), 1, (size_t)n, f) == (size_t)n;
    std::fclose(f);
    if (!good) set_error(std::string("short read of ") + path);
    return good;
}

struct Page {
    uint32_t w = 0, h = 0, bits = 0, fmt = 1, spp = 1, comp = 1, planar = 1, rows_per_strip = 0xffffffffu;
    std::vector<uint32_t> offsets, counts;
};

// Values of one IFD entry (SHORT or LONG, any count).
bool entry_values(const Reader &r, size_t e, std::vector<uint32_t> &vals) {
    const uint16_t type = r.u16(e + 2);
    const uint32_t count = r.u32(e + 4);
    const size_t size = type == 3 ? 2 : (type == 4 ? 4 : (type == 1 ? 1 : 0));
    if (!size) return false;
    if (count > (1u << 28)) return false;
    const size_t total = size * count;
    size_t at = e + 8;
    if (total > 4) {
        at = r.u32(e + 8);
        if (!r.ok(at, total)) return false;
    }
    vals.resize(count);
    for (uint32_t k = 0; k < count; ++k)
        vals[k] = type == 3 ? r.u16(at + 2 * k) : (type == 4 ? r.u32(at + 4 * k) : r.buf[at + k]);
    return true;
}

float sample(const Reader &r, size_t o, const Page &p) {
    switch (p.bits) {
    case 8:
        return p.fmt == 2 ? (float)(int8_t)r.buf[o] : (float)r.buf[o];
    case 16:
        return p.fmt == 2 ? (float)(int16_t)r.u16(o) : (float)r.u16(o);
    case 32: {
        const uint32_t b = r.u32(o);
        if (p.fmt == 3) {
            float f;
            std::memcpy(&f, &b, 4);
            return f;
        }
        return p.fmt == 2 ? (float)(int32_t)b : (float)b;
    }
    default: {  // 64-bit float
        const uint64_t b = r.u64(o);
        double v;
        std::memcpy(&v, &b, 8);
        return (float)v;
    }
    }
}

void put_u16(std::vector<unsigned char> &b, uint16_t v) {
    b.push_back(v & 0xff);
    b.push_back(v >> 8);
}
void put_u32(std::vector<unsigned char> &b, uint32_t v) {
    for (int k = 0; k < 4; ++k) b.push_back((v >> (8 * k)) & 0xff);
}

bool write_file(const char *path, const void *data, size_t n) {
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        set_error(std::string("cannot create ") + path + ": " + std::strerror(errno));
        return false;
    }
    const bool good = std::fwrite(data, 1, n, f) == n;
    if (std::fclose(f) != 0 || !good) {
        set_error(std::string("write failed: ") + path);
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

int stt_tiff_read(const char *path, int *w, int *h, int *d, float **data) {
    if (!path || !w || !h || !d || !data) return set_error("null argument"), STT_ERR_INVALID;
    *data = nullptr;
    Reader r;
    if (!read_file(path, r.buf)) return STT_ERR_INVALID;
    if (r.buf.size() < 8 || !((r.buf[0] == 'I' && r.buf[1] == 'I') || (r.buf[0] == 'M' && r.buf[1] == 'M')))
        return set_error(std::string(path) + ": not a TIFF file"), STT_ERR_INVALID;
    r.be = r.buf[0] == 'M';
    if (r.u16(2) != 42) return set_error(std::string(path) + ": not a classic TIFF (BigTIFF is not read)"), STT_ERR_INVALID;
    std::vector<Page> pages;
    uint32_t ifd = r.u32(4);
    while (ifd) {
        if (!r.ok(ifd, 2) || pages.size() > 1000000) return set_error(std::string(path) + ": bad IFD offset"), STT_ERR_INVALID;
        const uint16_t n = r.u16(ifd);
        if (!r.ok(ifd + 2, 12u * n + 4)) return set_error(std::string(path) + ": truncated IFD"), STT_ERR_INVALID;
        Page p;
        for (uint16_t k = 0; k < n; ++k) {
            const size_t e = ifd + 2 + 12u * k;
            const uint16_t tag = r.u16(e);
            std::vector<uint32_t> v;
            if (!entry_values(r, e, v) || v.empty()) continue;
            switch (tag) {
            case 256: p.w = v[0]; break;
            case 257: p.h = v[0]; break;
            case 258: p.bits = v[0]; break;
            case 259: p.comp = v[0]; break;
            case 273: p.offsets = v; break;
            case 277: p.spp = v[0]; break;
            case 278: p.rows_per_strip = v[0]; break;
            case 279: p.counts = v; break;
            case 284: p.planar = v[0]; break;
            case 339: p.fmt = v[0]; break;
            case 322: return set_error(std::string(path) + ": tiled TIFF is not supported"), STT_ERR_UNSUPPORTED;
            default: break;
            }
        }
        if (p.comp != 1) return set_error(std::string(path) + ": compressed TIFF is not supported"), STT_ERR_UNSUPPORTED;
        if (p.spp != 1) return set_error(std::string(path) + ": one sample per pixel expected"), STT_ERR_UNSUPPORTED;
        const bool fmt_ok = (p.fmt == 1 || p.fmt == 2) ? (p.bits == 8 || p.bits == 16 || p.bits == 32)
                                                         : (p.fmt == 3 && (p.bits == 32 || p.bits == 64));
        if (!fmt_ok) return set_error(std::string(path) + ": unsupported sample type"), STT_ERR_UNSUPPORTED;
        if (!p.w || !p.h || p.offsets.empty()) return set_error(std::string(path) + ": missing image tags"), STT_ERR_INVALID;
        pages.push_back(p);
        ifd = r.u32(ifd + 2 + 12u * n);
    }
    if (pages.empty()) return set_error(std::string(path) + ": no image"), STT_ERR_INVALID;
    const Page &p0 = pages[0];
    for (const Page &p : pages)
        if (p.w != p0.w || p.h != p0.h) return set_error(std::string(path) + ": pages differ in size"), STT_ERR_UNSUPPORTED;
    const size_t plane = (size_t)p0.w * p0.h;
    float *out = static_cast<float *>(std::malloc(sizeof(float) * plane * pages.size()));
    if (!out) return set_error("out of host memory"), STT_ERR_NOMEM;
    for (size_t z = 0; z < pages.size(); ++z) {
        const Page &p = pages[z];
        const size_t bps = p.bits / 8;
        const uint32_t rps = p.rows_per_strip == 0 ? p.h : std::min(p.rows_per_strip, p.h);
        size_t px = 0;
        for (size_t s = 0; s < p.offsets.size() && px < plane; ++s) {
            const size_t rows = std::min<size_t>(rps, p.h - s * rps);
            const size_t n = rows * p.w;
            if (!r.ok(p.offsets[s], n * bps)) {
                std::free(out);
                return set_error(std::string(path) + ": strip outside the file"), STT_ERR_INVALID;
            }
            for (size_t q = 0; q < n; ++q) out[z * plane + px + q] = sample(r, p.offsets[s] + q * bps, p);
            px += n;
        }
        if (px != plane) {
            std::free(out);
            return set_error(std::string(path) + ": strips do not cover the image"), STT_ERR_INVALID;
        }
    }
    *w = (int)p0.w;
    *h = (int)p0.h;
    *d = (int)pages.size();
    *data = out;
    return STT_OK;
}

int stt_tiff_write(const char *path, int w, int h, int d, const float *data) {
    if (!path || !data || w < 1 || h < 1 || d < 1) return set_error("bad arguments"), STT_ERR_INVALID;
    const size_t plane = (size_t)w * h * 4;
    const size_t nent = 11, ifd_size = 2 + 12 * nent + 4;
    if ((8 + (plane + ifd_size) * (size_t)d) >> 32)
        return set_error("stack too large for a classic TIFF (4 GiB)"), STT_ERR_INVALID;
    std::vector<unsigned char> b;
    b.reserve(8 + (plane + ifd_size) * d);
    b.push_back('I');
    b.push_back('I');
    put_u16(b, 42);
    put_u32(b, 8);
    for (int z = 0; z < d; ++z) {
        const uint32_t ifd = (uint32_t)b.size();
        const uint32_t data_at = ifd + (uint32_t)ifd_size;
        const uint32_t next = z + 1 < d ? data_at + (uint32_t)plane : 0;
        put_u16(b, (uint16_t)nent);
        auto entry = [&](uint16_t tag, uint16_t type, uint32_t value) {
            put_u16(b, tag);
            put_u16(b, type);
            put_u32(b, 1);
            if (type == 3) {
                put_u16(b, (uint16_t)value);
                put_u16(b, 0);
            } else {
                put_u32(b, value);
            }
        };
        entry(256, 4, (uint32_t)w);           // ImageWidth
        entry(257, 4, (uint32_t)h);           // ImageLength
        entry(258, 3, 32);                    // BitsPerSample
        entry(259, 3, 1);                     // Compression: none
        entry(262, 3, 1);                     // Photometric: black is zero
        entry(273, 4, data_at);               // StripOffsets
        entry(277, 3, 1);                     // SamplesPerPixel
        entry(278, 4, (uint32_t)h);           // RowsPerStrip: one strip
        entry(279, 4, (uint32_t)plane);       // StripByteCounts
        entry(284, 3, 1);                     // PlanarConfiguration: chunky
        entry(339, 3, 3);                     // SampleFormat: IEEE float
        put_u32(b, next);
        const unsigned char *src = reinterpret_cast<const unsigned char *>(data + (size_t)z * w * h);
        b.insert(b.end(), src, src + plane);  // x86 and aarch64 hosts are little endian
    }
    return write_file(path, b.data(), b.size()) ? STT_OK : STT_ERR_INVALID;
}

int stt_analyze_write(const char *hdr_path, int w, int h, int d, int c, const float *data) {
    if (!hdr_path || !data || w < 1 || h < 1 || d < 1 || c < 1) return set_error("bad arguments"), STT_ERR_INVALID;
    std::string hp(hdr_path);
    if (hp.size() < 4 || hp.compare(hp.size() - 4, 4, ".hdr") != 0)
        return set_error("Analyze header path must end in .hdr"), STT_ERR_INVALID;
    const std::string ip = hp.substr(0, hp.size() - 4) + ".img";
    unsigned char hdr[348];
    std::memset(hdr, 0, sizeof(hdr));
    auto i32 = [&](int off, int32_t v) { std::memcpy(hdr + off, &v, 4); };
    auto i16 = [&](int off, int16_t v) { std::memcpy(hdr + off, &v, 2); };
    auto f32 = [&](int off, float v) { std::memcpy(hdr + off, &v, 4); };
    i32(0, 348);              // sizeof_hdr
    i32(32, 16384);           // extents
    hdr[38] = 'r';            // regular
    i16(40, 4);               // dim[0]
    i16(42, (int16_t)w);      // dim[1..4]
    i16(44, (int16_t)h);
    i16(46, (int16_t)d);
    i16(48, (int16_t)c);
    i16(70, 16);              // datatype: float
    i16(72, 32);              // bitpix
    f32(80, 1.0f);            // pixdim[1..3]
    f32(84, 1.0f);
    f32(88, 1.0f);
    f32(112, 1.0f);           // funused1: scale factor
    if (w > 32767 || h > 32767 || d > 32767 || c > 32767)
        return set_error("Analyze extents are 16-bit"), STT_ERR_INVALID;
    if (!write_file(hdr_path, hdr, sizeof(hdr))) return STT_ERR_INVALID;
    return write_file(ip.c_str(), data, sizeof(float) * (size_t)w * h * d * c) ? STT_OK : STT_ERR_INVALID;
}

int stt_analyze_read(const char *hdr_path, int *w, int *h, int *d, int *c, float **data) {
    if (!hdr_path || !w || !h || !d || !c || !data) return set_error("null argument"), STT_ERR_INVALID;
    *data = nullptr;
    std::vector<unsigned char> hdr;
    if (!read_file(hdr_path, hdr)) return STT_ERR_INVALID;
    int32_t sz;
    if (hdr.size() < 348 || (std::memcpy(&sz, hdr.data(), 4), sz != 348))
        return set_error(std::string(hdr_path) + ": not a little-endian Analyze header"), STT_ERR_INVALID;
    int16_t dim[5], dt;
    std::memcpy(dim, hdr.data() + 40, 10);
    std::memcpy(&dt, hdr.data() + 70, 2);
    if (dt != 16) return set_error(std::string(hdr_path) + ": only float Analyze data is read"), STT_ERR_UNSUPPORTED;
    const int ew = dim[1], eh = dim[0] >= 2 ? dim[2] : 1, ed = dim[0] >= 3 ? dim[3] : 1, ec = dim[0] >= 4 ? dim[4] : 1;
    if (ew < 1 || eh < 1 || ed < 1 || ec < 1) return set_error(std::string(hdr_path) + ": bad extents"), STT_ERR_INVALID;
    std::string ip(hdr_path);
    ip = ip.substr(0, ip.size() - 4) + ".img";
    std::vector<unsigned char> img;
    if (!read_file(ip.c_str(), img)) return STT_ERR_INVALID;
    const size_t n = (size_t)ew * eh * ed * ec;
    if (img.size() < n * 4) return set_error(ip + ": shorter than the header says"), STT_ERR_INVALID;
    float *out = static_cast<float *>(std::malloc(n * 4));
    if (!out) return set_error("out of host memory"), STT_ERR_NOMEM;
    std::memcpy(out, img.data(), n * 4);
    *w = ew;
    *h = eh;
    *d = ed;
    *c = ec;
    *data = out;
    return STT_OK;
}

void stt_host_free(void *p) { std::free(p); }

}  // extern "C"
