// Headless image output.  The reference shows its frames through an OpenGL
// pixel buffer object (core/utilities.h:110-153, app/opengl_display.cpp);
// gs_b200 renders into plain RGBA8 buffers (row 0 = bottom, as in that
// buffer) and writes them to files, top row first: binary PPM (P6, RGB) or
// PNG (8-bit RGBA, the zlib stream made of stored deflate blocks, so no
// compression library is needed).
#include "../../include/gs_b200.h"

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

// CRC-32 of the PNG chunks (ISO 3309 / ITU-T V.42 polynomial, reflected)
struct CrcTable {
    uint32_t t[256];
    CrcTable()
    {
        for (uint32_t n = 0; n < 256; ++n) {
            uint32_t c = n;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[n] = c;
        }
    }
};

uint32_t crc_update(uint32_t crc, const uint8_t* p, size_t n)
{
    static const CrcTable tab;
    for (size_t i = 0; i < n; ++i) crc = tab.t[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<uint8_t>& b, uint32_t v)
{
    b.push_back((uint8_t)(v >> 24));
    b.push_back((uint8_t)(v >> 16));
    b.push_back((uint8_t)(v >> 8));
    b.push_back((uint8_t)v);
}

bool write_chunk(FILE* f, const char type[4], const std::vector<uint8_t>& data)
{
    std::vector<uint8_t> head;
    put_be32(head, (uint32_t)data.size());
    head.insert(head.end(), type, type + 4);
    uint32_t crc = crc_update(0xFFFFFFFFu, reinterpret_cast<const uint8_t*>(type), 4);
    crc = crc_update(crc, data.data(), data.size()) ^ 0xFFFFFFFFu;
    std::vector<uint8_t> tail;
    put_be32(tail, crc);
    return std::fwrite(head.data(), 1, head.size(), f) == head.size() &&
           (data.empty() || std::fwrite(data.data(), 1, data.size(), f) == data.size()) &&
           std::fwrite(tail.data(), 1, tail.size(), f) == tail.size();
}

bool valid(const char* path, const uint8_t* rgba, int32_t w, int32_t h)
{
    return path && rgba && w > 0 && h > 0 && w <= 65536 && h <= 65536;
}

}  // namespace

extern "C" {

GS_API int gs_write_ppm(const char* path, const uint8_t* h_rgba, int32_t width, int32_t height)
{
    if (!valid(path, h_rgba, width, height)) return GS_ERR_INVALID;
    FILE* f = std::fopen(path, "wb");
    if (!f) return GS_ERR_INVALID;
    std::fprintf(f, "P6\n%d %d\n255\n", width, height);
    std::vector<uint8_t> row(3 * (size_t)width);
    bool ok = true;
    for (int32_t y = height - 1; y >= 0 && ok; --y) {
        const uint8_t* src = h_rgba + 4 * (size_t)width * y;
        for (int32_t x = 0; x < width; ++x) std::memcpy(&row[3 * (size_t)x], src + 4 * (size_t)x, 3);
        ok = std::fwrite(row.data(), 1, row.size(), f) == row.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GS_OK : GS_ERR_INVALID;
}

GS_API int gs_write_png(const char* path, const uint8_t* h_rgba, int32_t width, int32_t height)
{
    if (!valid(path, h_rgba, width, height)) return GS_ERR_INVALID;
    // filtered scanlines: filter type 0, then the row's RGBA bytes, top row first
    const size_t stride = 4 * (size_t)width;
    std::vector<uint8_t> raw((stride + 1) * (size_t)height);
    for (int32_t r = 0; r < height; ++r) {
        uint8_t* dst = raw.data() + (stride + 1) * (size_t)r;
        dst[0] = 0;
        std::memcpy(dst + 1, h_rgba + stride * (size_t)(height - 1 - r), stride);
    }
    // zlib stream (RFC 1950): header, stored deflate blocks (RFC 1951), Adler-32
    std::vector<uint8_t> z;
    z.reserve(raw.size() + raw.size() / 65535 * 5 + 16);
    z.push_back(0x78);
    z.push_back(0x01);
    uint32_t a = 1, b = 0;
    for (size_t off = 0; off < raw.size() || off == 0;) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)len);
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len);
        z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + (ptrdiff_t)off, raw.begin() + (ptrdiff_t)(off + len));
        for (size_t i = off; i < off + len; ++i) {
            a = (a + raw[i]) % 65521u;
            b = (b + a) % 65521u;
        }
        off += len;
        if (last) break;
    }
    put_be32(z, (b << 16) | a);

    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    const uint8_t rest[5] = {8, 6, 0, 0, 0};  // 8 bits, RGBA, deflate, filter set 0, no interlace
    ihdr.insert(ihdr.end(), rest, rest + 5);

    FILE* f = std::fopen(path, "wb");
    if (!f) return GS_ERR_INVALID;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    bool ok = std::fwrite(sig, 1, 8, f) == 8 && write_chunk(f, "IHDR", ihdr) && write_chunk(f, "IDAT", z) &&
              write_chunk(f, "IEND", {});
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GS_OK : GS_ERR_INVALID;
}

}  // extern "C"
