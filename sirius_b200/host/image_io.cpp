// image_io.cpp — image output of headless frame buffers: PNG (8-bit sRGB),
// OpenEXR (half-float, ZIP-compressed scanlines), PFM and PPM.
//
// The pixel conversions follow the reference's output drivers:
//   - PNG (PNGWriter::writeRGB / writeRGBA, OUPN001A.cpp:45-97): each colour
//     channel through toSRGB8 (OUPN001A.h:154-163: clamp to [0, 1], the sRGB
//     curve 12.92 x below 0.0031308 else 1.055 x^(1/2.4) - 0.055, then
//     x * 255 + 0.5 clamped and truncated), alpha as linear x * 255 + 0.5;
//   - EXR (EXRWriter::writeEXR, OUEW001A.cpp:17-195): channels B, G, R (and A
//     first for RGBA) stored as HALF, ZIP compression, no metadata attributes;
//   - PFM / PPM (OUEW001A.h:94-124): PF, bottom row first, little-endian
//     floats; P6 with the toSRGB8 bytes.
// The containers are written here from the PNG and OpenEXR file-format
// specifications; zlib does the deflate. A decoder sees the same pixel values
// as in the reference's files (the compressed bytes may differ).
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "sirius_cuda.h"

namespace {

uint8_t to_srgb8(float linear) {
    const float c = std::clamp(linear, 0.0f, 1.0f);
    const float s = c <= 0.0031308f ? 12.92f * c : 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
    return static_cast<uint8_t>(std::clamp(s * 255.0f + 0.5f, 0.0f, 255.0f));
}

uint8_t to_linear8(float x) { return static_cast<uint8_t>(std::clamp(x * 255.0f + 0.5f, 0.0f, 255.0f)); }

// binary32 -> binary16 as the reference's EXR files hold them (tinyexr's
// conversion behind EXRWriter): the magnitude rounds half away from zero on the
// first dropped bit, overflow gives infinity, every NaN becomes the quiet NaN
// 0x7e00, and binary32 subnormals flush to zero.
uint16_t to_half(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t exp = (u >> 23) & 0xffu, man = u & 0x7fffffu;
    if (exp == 0) return uint16_t(sign);
    if (exp == 0xffu) return uint16_t(sign | 0x7c00u | (man ? 0x200u : 0u));
    const int e = int(exp) - 127 + 15;
    if (e >= 31) return uint16_t(sign | 0x7c00u);
    if (e <= 0) {  // a half subnormal, or zero below 2^-25
        if (14 - e > 24) return uint16_t(sign);
        const uint32_t m = man | 0x800000u;
        uint32_t h = m >> (14 - e);
        if ((m >> (13 - e)) & 1u) ++h;
        return uint16_t(sign | h);
    }
    uint32_t h = (uint32_t(e) << 10) | (man >> 13);
    if (man & 0x1000u) ++h;  // a carry into the exponent is the right result (up to infinity)
    return uint16_t(sign | h);
}

void put_be32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back(uint8_t(x >> 24)); v.push_back(uint8_t(x >> 16)); v.push_back(uint8_t(x >> 8)); v.push_back(uint8_t(x));
}
template <class T>
void put_le(std::vector<uint8_t>& v, T x) {
    uint8_t b[sizeof(T)];
    std::memcpy(b, &x, sizeof(T));
    v.insert(v.end(), b, b + sizeof(T));
}

bool deflate_bytes(const uint8_t* in, size_t n, std::vector<uint8_t>& out) {
    uLongf cap = compressBound(uLong(n));
    out.resize(cap);
    if (compress2(out.data(), &cap, in, uLong(n), 6) != Z_OK) return false;
    out.resize(cap);
    return true;
}

bool write_file(const char* path, const std::vector<uint8_t>& bytes) {
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return false;
    const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), fp) == bytes.size();
    return (std::fclose(fp) == 0) && ok;
}

void png_chunk(std::vector<uint8_t>& f, const char* type, const std::vector<uint8_t>& data) {
    put_be32(f, uint32_t(data.size()));
    const size_t start = f.size();
    f.insert(f.end(), type, type + 4);
    f.insert(f.end(), data.begin(), data.end());
    put_be32(f, uint32_t(crc32(0L, f.data() + start, uInt(f.size() - start))));
}

int write_png(const char* path, int w, int h, int channels, const float* px) {
    if (!path || !px || w <= 0 || h <= 0 || (channels != 3 && channels != 4)) return SIRIUS_ERR_INVALID_ARGUMENT;
    const size_t row = size_t(w) * channels;
    std::vector<uint8_t> raw((row + 1) * size_t(h));
    for (int y = 0; y < h; ++y) {
        uint8_t* r = raw.data() + (row + 1) * size_t(y);
        r[0] = 0;  // filter type None
        for (int x = 0; x < w; ++x) {
            const float* p = px + (size_t(y) * w + x) * channels;
            for (int c = 0; c < 3; ++c) r[1 + size_t(x) * channels + c] = to_srgb8(p[c]);
            if (channels == 4) r[1 + size_t(x) * 4 + 3] = to_linear8(p[3]);
        }
    }
    std::vector<uint8_t> z;
    if (!deflate_bytes(raw.data(), raw.size(), z)) return SIRIUS_ERR_OUT_OF_MEMORY;
    std::vector<uint8_t> f = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, uint32_t(w));
    put_be32(ihdr, uint32_t(h));
    ihdr.push_back(8);                          // bit depth
    ihdr.push_back(channels == 4 ? 6 : 2);      // colour type RGBA / RGB
    ihdr.push_back(0); ihdr.push_back(0); ihdr.push_back(0);
    png_chunk(f, "IHDR", ihdr);
    png_chunk(f, "IDAT", z);
    png_chunk(f, "IEND", {});
    return write_file(path, f) ? SIRIUS_OK : SIRIUS_ERR_INVALID_ARGUMENT;
}

void exr_attr(std::vector<uint8_t>& f, const char* name, const char* type, const std::vector<uint8_t>& value) {
    f.insert(f.end(), name, name + std::strlen(name) + 1);
    f.insert(f.end(), type, type + std::strlen(type) + 1);
    put_le<int32_t>(f, int32_t(value.size()));
    f.insert(f.end(), value.begin(), value.end());
}

int write_exr(const char* path, int w, int h, int channels, const float* px) {
    if (!path || !px || w <= 0 || h <= 0 || (channels != 3 && channels != 4)) return SIRIUS_ERR_INVALID_ARGUMENT;
    // file channel order (alphabetical): A (RGBA only), B, G, R -> source component
    std::vector<int> comp = channels == 4 ? std::vector<int>{3, 2, 1, 0} : std::vector<int>{2, 1, 0};
    const char* names4[4] = {"A", "B", "G", "R"};
    const char* names3[3] = {"B", "G", "R"};
    std::vector<uint8_t> f = {0x76, 0x2f, 0x31, 0x01, 2, 0, 0, 0};
    std::vector<uint8_t> chl;
    for (int c = 0; c < channels; ++c) {
        const char* n = channels == 4 ? names4[c] : names3[c];
        chl.insert(chl.end(), n, n + std::strlen(n) + 1);
        put_le<int32_t>(chl, 1);           // HALF
        chl.push_back(0); chl.push_back(0); chl.push_back(0); chl.push_back(0);  // pLinear, reserved
        put_le<int32_t>(chl, 1);
        put_le<int32_t>(chl, 1);           // x / y sampling
    }
    chl.push_back(0);
    exr_attr(f, "channels", "chlist", chl);
    exr_attr(f, "compression", "compression", {3});  // ZIP, 16 scanlines per chunk
    std::vector<uint8_t> box;
    put_le<int32_t>(box, 0); put_le<int32_t>(box, 0); put_le<int32_t>(box, w - 1); put_le<int32_t>(box, h - 1);
    exr_attr(f, "dataWindow", "box2i", box);
    exr_attr(f, "displayWindow", "box2i", box);
    exr_attr(f, "lineOrder", "lineOrder", {0});
    std::vector<uint8_t> one;
    put_le<float>(one, 1.0f);
    exr_attr(f, "pixelAspectRatio", "float", one);
    std::vector<uint8_t> ctr;
    put_le<float>(ctr, 0.0f); put_le<float>(ctr, 0.0f);
    exr_attr(f, "screenWindowCenter", "v2f", ctr);
    exr_attr(f, "screenWindowWidth", "float", one);
    f.push_back(0);
    const int lines = 16, n_chunks = (h + lines - 1) / lines;
    const size_t table = f.size();
    f.resize(f.size() + 8 * size_t(n_chunks));
    std::vector<uint8_t> raw, pred, z;
    for (int k = 0; k < n_chunks; ++k) {
        const int y0 = k * lines, y1 = std::min(h, y0 + lines);
        raw.clear();
        for (int y = y0; y < y1; ++y)
            for (int c = 0; c < channels; ++c)
                for (int x = 0; x < w; ++x) put_le<uint16_t>(raw, to_half(px[(size_t(y) * w + x) * channels + comp[c]]));
        // ZIP: bytes split into even / odd halves, then a byte-wise delta predictor
        const size_t n = raw.size(), half = (n + 1) / 2;
        pred.resize(n);
        for (size_t i = 0; i < n; ++i) pred[(i & 1) ? half + i / 2 : i / 2] = raw[i];
        for (size_t i = n; i-- > 1;) pred[i] = uint8_t(int(pred[i]) - int(pred[i - 1]) + 128);
        if (!deflate_bytes(pred.data(), n, z)) return SIRIUS_ERR_OUT_OF_MEMORY;
        const std::vector<uint8_t>& body = z.size() < n ? z : raw;  // stored raw when deflate does not shrink it
        const uint64_t off = uint64_t(f.size());
        std::memcpy(f.data() + table + 8 * size_t(k), &off, 8);
        put_le<int32_t>(f, y0);
        put_le<int32_t>(f, int32_t(body.size()));
        f.insert(f.end(), body.begin(), body.end());
    }
    return write_file(path, f) ? SIRIUS_OK : SIRIUS_ERR_INVALID_ARGUMENT;
}

}  // namespace

extern "C" {

int sirius_cuda_write_png(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels) {
    return write_png(path, width, height, channels, pixels);
}

int sirius_cuda_write_exr(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels) {
    return write_exr(path, width, height, channels, pixels);
}

int sirius_cuda_write_pfm(const char* path, int32_t width, int32_t height, const float* rgb) {
    if (!path || !rgb || width <= 0 || height <= 0) return SIRIUS_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> f;
    const std::string head = "PF\n" + std::to_string(width) + " " + std::to_string(height) + "\n-1.0\n";
    f.insert(f.end(), head.begin(), head.end());
    for (int y = height - 1; y >= 0; --y)
        for (int x = 0; x < width * 3; ++x) put_le<float>(f, rgb[size_t(y) * width * 3 + x]);
    return write_file(path, f) ? SIRIUS_OK : SIRIUS_ERR_INVALID_ARGUMENT;
}

int sirius_cuda_write_ppm(const char* path, int32_t width, int32_t height, const float* rgb) {
    if (!path || !rgb || width <= 0 || height <= 0) return SIRIUS_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> f;
    const std::string head = "P6\n" + std::to_string(width) + " " + std::to_string(height) + "\n255\n";
    f.insert(f.end(), head.begin(), head.end());
    for (size_t i = 0; i < size_t(width) * height * 3; ++i) f.push_back(to_srgb8(rgb[i]));
    return write_file(path, f) ? SIRIUS_OK : SIRIUS_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
