// Image files from the output buffer: a tone-mapped 8-bit PNG and a linear
// half-float OpenEXR, as the reference's host program saves a render
// (HostProgram/main.cpp:120-168 saveOutputBufferAsImageFile, with
// HostProgram/image.cpp:193-256 writePNG / writeEXR).  Host code only; the
// encoders are written here from the PNG (RFC 2083, zlib RFC 1950, deflate
// RFC 1951 stored blocks) and OpenEXR (scanline file layout) specifications.
#include "../../include/vlrb.h"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

// sRGB_gamma_s (HostProgram/main.cpp:54-59).
float srgbGamma(float v) {
    if (v <= 0.0031308f) return 12.92f * v;
    return 1.055f * std::pow(v, 1.0f / 2.4f) - 0.055f;
}

// The host program's tone mapping: clamp at 0, scale by the brightness
// coefficient, 1 - exp(-x), sRGB gamma, x 256 truncated to 255
// (HostProgram/main.cpp:132-160).
uint8_t toneMap(float v, float brightness) {
    v = std::fmax(v, 0.0f);
    v *= brightness;
    v = 1.0f - std::exp(-v);
    v = srgbGamma(v);
    return static_cast<uint8_t>(std::min<uint32_t>(static_cast<uint32_t>(v * 256), 255u));
}

uint32_t crc32(const uint8_t* p, size_t n, uint32_t crc = 0) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return ~crc;
}

void putBE32(std::vector<uint8_t> &v, uint32_t x) {
    v.push_back(static_cast<uint8_t>(x >> 24));
    v.push_back(static_cast<uint8_t>(x >> 16));
    v.push_back(static_cast<uint8_t>(x >> 8));
    v.push_back(static_cast<uint8_t>(x));
}

void pngChunk(std::vector<uint8_t> &out, const char type[4], const std::vector<uint8_t> &data) {
    putBE32(out, static_cast<uint32_t>(data.size()));
    std::vector<uint8_t> td(type, type + 4);
    td.insert(td.end(), data.begin(), data.end());
    out.insert(out.end(), td.begin(), td.end());
    putBE32(out, crc32(td.data(), td.size()));
}

// RGBA8 PNG: filter 0 on every row, the zlib stream of stored deflate blocks.
bool writePng(const std::string &path, uint32_t w, uint32_t h, const std::vector<uint8_t> &rgba) {
    std::vector<uint8_t> raw;
    raw.reserve(size_t(h) * (size_t(w) * 4 + 1));
    for (uint32_t y = 0; y < h; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgba.begin() + size_t(y) * w * 4, rgba.begin() + size_t(y + 1) * w * 4);
    }
    std::vector<uint8_t> z = { 0x78, 0x01 };
    size_t pos = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + len == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(static_cast<uint8_t>(len));
        z.push_back(static_cast<uint8_t>(len >> 8));
        z.push_back(static_cast<uint8_t>(~len));
        z.push_back(static_cast<uint8_t>(~len >> 8));
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + len);
        pos += len;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;   // Adler-32
    for (uint8_t c : raw) {
        a = (a + c) % 65521u;
        b = (b + a) % 65521u;
    }
    putBE32(z, (b << 16) | a);
    std::vector<uint8_t> out = { 0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n' };
    std::vector<uint8_t> ihdr;
    putBE32(ihdr, w);
    putBE32(ihdr, h);
    ihdr.insert(ihdr.end(), { 8, 6, 0, 0, 0 });   // 8 bits, RGBA, deflate, filter 0, no interlace
    pngChunk(out, "IHDR", ihdr);
    pngChunk(out, "IDAT", z);
    pngChunk(out, "IEND", {});
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
    return std::fclose(f) == 0 && ok;
}

template <typename T> void putLE(std::vector<uint8_t> &v, T x) {
    uint8_t b[sizeof(T)];
    std::memcpy(b, &x, sizeof(T));
    v.insert(v.end(), b, b + sizeof(T));
}

void exrAttr(std::vector<uint8_t> &v, const char* name, const char* type, const std::vector<uint8_t> &value) {
    v.insert(v.end(), name, name + std::strlen(name) + 1);
    v.insert(v.end(), type, type + std::strlen(type) + 1);
    putLE<int32_t>(v, static_cast<int32_t>(value.size()));
    v.insert(v.end(), value.begin(), value.end());
}

// Scanline OpenEXR, no compression, channels A, B, G, R stored as half
// (the reference saves float RGBA as half, (A)BGR order), one line per block.
bool writeExr(const std::string &path, uint32_t w, uint32_t h, const float* rgba) {
    std::vector<uint8_t> v;
    putLE<int32_t>(v, 20000630);
    putLE<int32_t>(v, 2);
    std::vector<uint8_t> ch;
    for (const char* name : { "A", "B", "G", "R" }) {
        ch.push_back(static_cast<uint8_t>(name[0]));
        ch.push_back(0);
        putLE<int32_t>(ch, 1);           // HALF
        ch.insert(ch.end(), { 0, 0, 0, 0 });   // pLinear, reserved
        putLE<int32_t>(ch, 1);
        putLE<int32_t>(ch, 1);
    }
    ch.push_back(0);
    exrAttr(v, "channels", "chlist", ch);
    exrAttr(v, "compression", "compression", { 0 });
    std::vector<uint8_t> box;
    for (int32_t x : { 0, 0, static_cast<int32_t>(w) - 1, static_cast<int32_t>(h) - 1 }) putLE<int32_t>(box, x);
    exrAttr(v, "dataWindow", "box2i", box);
    exrAttr(v, "displayWindow", "box2i", box);
    exrAttr(v, "lineOrder", "lineOrder", { 0 });
    std::vector<uint8_t> one;
    putLE<float>(one, 1.0f);
    exrAttr(v, "pixelAspectRatio", "float", one);
    std::vector<uint8_t> center;
    putLE<float>(center, 0.0f);
    putLE<float>(center, 0.0f);
    exrAttr(v, "screenWindowCenter", "v2f", center);
    exrAttr(v, "screenWindowWidth", "float", one);
    v.push_back(0);
    const size_t lineBytes = size_t(w) * 4 * 2;
    const size_t tableAt = v.size();
    v.resize(v.size() + size_t(h) * 8);
    for (uint32_t y = 0; y < h; ++y) {
        const uint64_t offset = v.size();
        std::memcpy(v.data() + tableAt + size_t(y) * 8, &offset, 8);
        putLE<int32_t>(v, static_cast<int32_t>(y));
        putLE<int32_t>(v, static_cast<int32_t>(lineBytes));
        for (int c : { 3, 2, 1, 0 })
            for (uint32_t x = 0; x < w; ++x) {
                const __half hv = __float2half_rn(rgba[(size_t(y) * w + x) * 4 + c]);
                uint16_t bits;
                std::memcpy(&bits, &hv, 2);
                putLE<uint16_t>(v, bits);
            }
    }
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(v.data(), 1, v.size(), f) == v.size();
    return std::fclose(f) == 0 && ok;
}

} // namespace

extern "C" VLRResult vlrbWriteOutputImages(const float* rgba, uint32_t width, uint32_t height,
                                           const char* pathWithoutExtension, float brightnessCoeff) {
    if (!rgba || !pathWithoutExtension || width == 0 || height == 0) return VLRResult_InvalidArgument;
    try {
        std::vector<uint8_t> ldr(size_t(width) * height * 4);
        for (size_t i = 0; i < size_t(width) * height; ++i) {
            for (int c = 0; c < 3; ++c) ldr[i * 4 + c] = toneMap(rgba[i * 4 + c], brightnessCoeff);
            ldr[i * 4 + 3] = 0xFF;
        }
        const std::string base(pathWithoutExtension);
        if (!writePng(base + ".png", width, height, ldr)) return VLRResult_InternalError;
        if (!writeExr(base + ".exr", width, height, rgba)) return VLRResult_InternalError;
        return VLRResult_NoError;
    }
    catch (...) {
        return VLRResult_InternalError;
    }
}
