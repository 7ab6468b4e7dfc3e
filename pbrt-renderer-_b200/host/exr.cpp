// exr.cpp — OpenEXR writer for linear HDR films.
//
// The reference saves its accumulation buffer as a linear scene-referred
// EXR for comparison against Mitsuba (validation_tests/compare_exr.py reads
// it).  This writer produces the simplest valid OpenEXR 2 file: single part,
// scanline, no compression, three 32-bit float channels.  Layout (from the
// published OpenEXR file-layout document):
//   magic 0x762f3101, version 2 (no flags);
//   header: attributes (name\0 type\0 int32 size, value), ended by a 0 byte —
//     channels (chlist, channel names in ascending order: B, G, R),
//     compression (0 = none), dataWindow / displayWindow (box2i),
//     lineOrder (0 = increasing y), pixelAspectRatio (1),
//     screenWindowCenter (0, 0), screenWindowWidth (1);
//   line offset table: one uint64 file offset per scanline;
//   scanlines: int32 y, int32 byte count, then each channel's W values.
// All integers and floats little-endian.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "nori/nori.h"

namespace nori {

namespace {
struct Buf {
    std::vector<unsigned char> b;
    void raw(const void *p, size_t n) {
        const unsigned char *c = static_cast<const unsigned char *>(p);
        b.insert(b.end(), c, c + n);
    }
    void str(const char *s) { raw(s, std::strlen(s) + 1); }
    void i32(int32_t v) { raw(&v, 4); }
    void u64(uint64_t v) { raw(&v, 8); }
    void f32(float v) { raw(&v, 4); }
    void attr(const char *name, const char *type, int32_t size) {
        str(name);
        str(type);
        i32(size);
    }
};
}  // namespace

// rgb: W * H * 3 floats, row 0 = top of the image.
void writeEXR(const std::string &path, int width, int height, const float *rgb) {
    if (width <= 0 || height <= 0 || !rgb) throw NoriException("writeEXR: empty image");
    Buf h;
    const uint32_t magic = 20000630u;  // bytes 76 2f 31 01 in little-endian order
    h.raw(&magic, 4);
    h.i32(2);
    // channels: per channel name\0, pixel type (2 = FLOAT), pLinear (u8) + 3
    // reserved bytes, x/y sampling (int32 1, 1); then a terminating 0 byte
    const char *names[3] = {"B", "G", "R"};
    h.attr("channels", "chlist", 3 * (2 + 16) + 1);
    for (const char *n : names) {
        h.str(n);
        h.i32(2);
        unsigned char plin[4] = {0, 0, 0, 0};
        h.raw(plin, 4);
        h.i32(1);
        h.i32(1);
    }
    unsigned char zero = 0;
    h.raw(&zero, 1);
    h.attr("compression", "compression", 1);
    h.raw(&zero, 1);
    for (const char *win : {"dataWindow", "displayWindow"}) {
        h.attr(win, "box2i", 16);
        h.i32(0);
        h.i32(0);
        h.i32(width - 1);
        h.i32(height - 1);
    }
    h.attr("lineOrder", "lineOrder", 1);
    h.raw(&zero, 1);
    h.attr("pixelAspectRatio", "float", 4);
    h.f32(1.0f);
    h.attr("screenWindowCenter", "v2f", 8);
    h.f32(0.0f);
    h.f32(0.0f);
    h.attr("screenWindowWidth", "float", 4);
    h.f32(1.0f);
    h.raw(&zero, 1);  // end of header
    const uint64_t lineBytes = (uint64_t)width * 3 * 4;
    const uint64_t first = h.b.size() + (uint64_t)height * 8;
    for (int y = 0; y < height; y++) h.u64(first + (uint64_t)y * (8 + lineBytes));
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) throw NoriException("writeEXR: cannot write \"" + path + "\"");
    bool ok = std::fwrite(h.b.data(), 1, h.b.size(), f) == h.b.size();
    std::vector<float> line((size_t)width * 3);
    for (int y = 0; y < height && ok; y++) {
        for (int c = 0; c < 3; c++)  // B, G, R planes
            for (int x = 0; x < width; x++) line[(size_t)c * width + x] = rgb[((size_t)y * width + x) * 3 + (2 - c)];
        int32_t hdr[2] = {y, (int32_t)lineBytes};
        ok = std::fwrite(hdr, 4, 2, f) == 2 && std::fwrite(line.data(), 4, line.size(), f) == line.size();
    }
    if (std::fclose(f) != 0 || !ok) throw NoriException("writeEXR: write to \"" + path + "\" failed");
}

}  // namespace nori
