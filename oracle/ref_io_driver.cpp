// ref_io_driver.cpp — C entry points around the reference's OWN image output
// drivers (PNGWriter, OUPN001A.cpp; EXRWriter, OUEW001A.cpp, with the stb and
// tinyexr libraries the reference vendors), compiled from the reference's
// sources where they lie, by oracle/Makefile, into oracle/_ref/.
//
// TEST INFRASTRUCTURE ONLY: the image-output parity tests write the same
// buffer with these and with the library's writers and compare the decoded
// pixels.
#include <cstdint>
#include <string>
#include <vector>

#include "OUEW001A.h"
#include "OUPN001A.h"

using namespace sirius::render;

extern "C" {

int ref_write_png(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels) {
    if (channels == 4) return PNGWriter::writeRGBA(path, width, height, pixels) ? 1 : 0;
    return PNGWriter::writeRGB(path, width, height, pixels) ? 1 : 0;
}

int ref_write_exr(const char* path, int32_t width, int32_t height, int32_t channels, const float* pixels) {
    const size_t n = size_t(width) * height;
    if (channels == 4) {
        ImageBufferRGBA b(width, height);
        for (size_t i = 0; i < 4 * n; ++i) b.pixels[i] = pixels[i];
        return EXRWriter::writeEXR(path, b) ? 1 : 0;
    }
    ImageBuffer b(width, height);
    for (size_t i = 0; i < 3 * n; ++i) b.pixels[i] = pixels[i];
    return EXRWriter::writeEXR(path, b) ? 1 : 0;
}

int ref_write_pfm(const char* path, int32_t width, int32_t height, const float* rgb) {
    ImageBuffer b(width, height);
    for (size_t i = 0; i < size_t(width) * height * 3; ++i) b.pixels[i] = rgb[i];
    return EXRWriter::writePFM(path, b) ? 1 : 0;
}

int ref_write_ppm(const char* path, int32_t width, int32_t height, const float* rgb) {
    ImageBuffer b(width, height);
    for (size_t i = 0; i < size_t(width) * height * 3; ++i) b.pixels[i] = rgb[i];
    return EXRWriter::writePPM(path, b) ? 1 : 0;
}

}  // extern "C"
