// tiff.cpp -- see tiff.h
#include "tiff.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>

namespace xpr {

namespace {

struct Reader {
    std::vector<uint8_t> buf;
    bool be = false;

    uint16_t u16(size_t off) const
    {
        if (off + 2 > buf.size()) throw std::runtime_error("truncated TIFF");
        return be ? (uint16_t)((buf[off] << 8) | buf[off + 1]) : (uint16_t)(buf[off] | (buf[off + 1] << 8));
    }
    uint32_t u32(size_t off) const
    {
        if (off + 4 > buf.size()) throw std::runtime_error("truncated TIFF");
        return be ? ((uint32_t)buf[off] << 24) | ((uint32_t)buf[off + 1] << 16) | ((uint32_t)buf[off + 2] << 8) | buf[off + 3]
                  : (uint32_t)buf[off] | ((uint32_t)buf[off + 1] << 8) | ((uint32_t)buf[off + 2] << 16) | ((uint32_t)buf[off + 3] << 24);
    }
};

struct Ifd {
    TiffInfo info;
    std::vector<uint32_t> offsets, counts;
};

// value(s) of one IFD entry of type SHORT (3) or LONG (4)
std::vector<uint32_t> entry_values(const Reader &r, size_t e)
{
    const uint16_t type = r.u16(e + 2);
    const uint32_t count = r.u32(e + 4);
    const size_t sz = type == 3 ? 2 : (type == 4 ? 4 : 0);
    if (!sz) throw std::runtime_error("unsupported TIFF field type");
    if ((uint64_t)count * sz > (1ull << 31)) throw std::runtime_error("corrupt TIFF field");
    size_t at = (count * sz <= 4) ? e + 8 : r.u32(e + 8);
    std::vector<uint32_t> v(count);
    for (uint32_t i = 0; i < count; ++i) v[i] = sz == 2 ? r.u16(at + 2 * i) : r.u32(at + 4 * i);
    return v;
}

Ifd parse(const Reader &r)
{
    if (r.buf.size() < 8) throw std::runtime_error("not a TIFF file");
    if (r.u16(2) != 42) throw std::runtime_error("not a TIFF file (magic)");
    size_t ifd = r.u32(4);
    const uint16_t n = r.u16(ifd);
    Ifd out;
    for (uint16_t k = 0; k < n; ++k) {
        const size_t e = ifd + 2 + 12 * (size_t)k;
        const uint16_t tag = r.u16(e);
        switch (tag) {
            case 256: out.info.width = entry_values(r, e)[0]; break;
            case 257: out.info.height = entry_values(r, e)[0]; break;
            case 258: out.info.bits = (uint16_t)entry_values(r, e)[0]; break;
            case 259: out.info.compression = (uint16_t)entry_values(r, e)[0]; break;
            case 273: out.offsets = entry_values(r, e); break;
            case 277: out.info.samples = (uint16_t)entry_values(r, e)[0]; break;
            case 279: out.counts = entry_values(r, e); break;
            case 339: out.info.sample_format = (uint16_t)entry_values(r, e)[0]; break;
            default: break;
        }
    }
    return out;
}

Reader load(const std::string &path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Corrupted or missing TIFF file: " + path);
    Reader r;
    r.buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    if (r.buf.size() < 8) throw std::runtime_error("Corrupted or missing TIFF file: " + path);
    if (r.buf[0] == 'I' && r.buf[1] == 'I') r.be = false;
    else if (r.buf[0] == 'M' && r.buf[1] == 'M') r.be = true;
    else throw std::runtime_error("not a TIFF file: " + path);
    return r;
}

}  // namespace

bool tiff_info(const std::string &path, TiffInfo *info, std::string *err)
{
    try {
        Reader r = load(path);
        *info = parse(r).info;
        return true;
    } catch (const std::exception &e) {
        if (err) *err = e.what();
        return false;
    }
}

std::vector<float> tiff_read_f32(const std::string &path, uint32_t *width, uint32_t *height)
{
    Reader r = load(path);
    Ifd d = parse(r);
    const TiffInfo &i = d.info;
    if (i.sample_format != 3 || i.bits != 32 || i.samples != 1)
        throw std::runtime_error("Trying to load a tiff with an incompatble format (should be floating-point 32bits): " + path);
    if (i.compression != 1) throw std::runtime_error("compressed TIFF is not supported: " + path);
    if (i.width == 0 || i.height == 0) throw std::runtime_error("Trying to load a tiff with an incorrect size: " + path);
    if (d.offsets.empty() || d.offsets.size() != d.counts.size()) throw std::runtime_error("TIFF without strips: " + path);
    const uint64_t need = (uint64_t)i.width * i.height * 4;
    std::vector<uint8_t> raw;
    raw.reserve(need);
    for (size_t s = 0; s < d.offsets.size() && raw.size() < need; ++s) {
        const uint64_t o = d.offsets[s], c = d.counts[s];
        if (o + c > r.buf.size()) throw std::runtime_error("truncated TIFF strip: " + path);
        raw.insert(raw.end(), r.buf.begin() + o, r.buf.begin() + o + c);
    }
    if (raw.size() < need) throw std::runtime_error("truncated TIFF data: " + path);
    std::vector<float> out((size_t)i.width * i.height);
    if (r.be) {
        for (size_t k = 0; k < out.size(); ++k) {
            uint8_t b[4] = {raw[4 * k + 3], raw[4 * k + 2], raw[4 * k + 1], raw[4 * k]};
            std::memcpy(&out[k], b, 4);
        }
    } else {
        std::memcpy(out.data(), raw.data(), need);
    }
    if (width) *width = i.width;
    if (height) *height = i.height;
    return out;
}

void tiff_write_f32(const std::string &path, const float *data, uint32_t width, uint32_t height)
{
    const uint32_t nbytes = width * height * 4u;
    const uint16_t n_entries = 10;
    const uint32_t ifd_off = 8;
    const uint32_t data_off = ifd_off + 2 + 12 * n_entries + 4;
    std::vector<uint8_t> b(data_off);
    auto w16 = [&](size_t at, uint16_t v) { b[at] = (uint8_t)v; b[at + 1] = (uint8_t)(v >> 8); };
    auto w32 = [&](size_t at, uint32_t v) { for (int k = 0; k < 4; ++k) b[at + k] = (uint8_t)(v >> (8 * k)); };
    b[0] = 'I'; b[1] = 'I';
    w16(2, 42);
    w32(4, ifd_off);
    w16(ifd_off, n_entries);
    size_t e = ifd_off + 2;
    auto entry = [&](uint16_t tag, uint16_t type, uint32_t value) {
        w16(e, tag); w16(e + 2, type); w32(e + 4, 1);
        if (type == 3) w16(e + 8, (uint16_t)value); else w32(e + 8, value);
        e += 12;
    };
    entry(256, 4, width);        // ImageWidth
    entry(257, 4, height);       // ImageLength
    entry(258, 3, 32);           // BitsPerSample
    entry(259, 3, 1);            // Compression: none
    entry(262, 3, 1);            // PhotometricInterpretation: BlackIsZero
    entry(273, 4, data_off);     // StripOffsets
    entry(277, 3, 1);            // SamplesPerPixel
    entry(278, 4, height);       // RowsPerStrip
    entry(279, 4, nbytes);       // StripByteCounts
    entry(339, 3, 3);            // SampleFormat: IEEE floating point
    w32(e, 0);                   // no next IFD
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("cannot write TIFF: " + path);
    f.write((const char *)b.data(), (std::streamsize)b.size());
    f.write((const char *)data, (std::streamsize)nbytes);
    if (!f) throw std::runtime_error("cannot write TIFF: " + path);
}

}  // namespace xpr
