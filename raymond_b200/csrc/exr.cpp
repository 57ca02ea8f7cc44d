// OpenEXR output of the film.  The reference saves frames with tinyexr's
// SaveEXR (utils/Metal.swift:75-126, called from Renderer.swift:806): four
// 32-bit float channels stored in the order A, B, G, R, alpha 1, each colour
// the film times a normalisation factor, ZIP-compressed unless the image is
// smaller than 16 x 16 in both directions.  This writer produces the same
// kind of file from the OpenEXR format description (single-part scanline
// image; ZIP: blocks of 16 scanlines, bytes split into even and odd halves,
// delta-coded, then deflated with zlib).
#include "exr.h"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace rmdhost {

namespace {

void put32(std::vector<unsigned char> &b, uint32_t v) {
    for (int k = 0; k < 4; k++) b.push_back((unsigned char)(v >> (8 * k)));
}
void putF(std::vector<unsigned char> &b, float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    put32(b, u);
}
void putStr(std::vector<unsigned char> &b, const char *s) {
    b.insert(b.end(), s, s + std::strlen(s) + 1);
}
// attribute: name, type name, byte size, value
void attribute(std::vector<unsigned char> &b, const char *name, const char *type,
               const std::vector<unsigned char> &value) {
    putStr(b, name);
    putStr(b, type);
    put32(b, (uint32_t)value.size());
    b.insert(b.end(), value.begin(), value.end());
}

// EXR ZIP preprocessing: bytes at even positions, then at odd positions,
// then each byte replaced by its difference to the previous one (+128, mod 256).
void zipPredict(const std::vector<unsigned char> &in, std::vector<unsigned char> &out) {
    const size_t n = in.size();
    out.resize(n);
    size_t a = 0, b = (n + 1) / 2;
    for (size_t i = 0; i < n; i += 2) {
        out[a++] = in[i];
        if (i + 1 < n) out[b++] = in[i + 1];
    }
    int prev = n ? out[0] : 0;
    for (size_t i = 1; i < n; i++) {
        const int cur = out[i];
        out[i] = (unsigned char)((cur - prev + 128 + 256) & 0xff);
        prev = cur;
    }
}

}  // namespace

std::string writeExrRgba(const char *path, const float *rgba, uint32_t width, uint32_t height, ExrCompression c) {
    if (!path || !rgba || width == 0 || height == 0) return "empty image or NULL argument";
    if (width > (1u << 30) / 16 || height > (1u << 30)) return "image too large for one EXR part";
    if (c == ExrCompression::Auto) c = (width < 16 && height < 16) ? ExrCompression::None : ExrCompression::Zip;
    const uint32_t linesPerChunk = c == ExrCompression::Zip ? 16u : 1u;
    const uint32_t chunks = (height + linesPerChunk - 1) / linesPerChunk;

    std::vector<unsigned char> file;
    put32(file, 20000630u);  // magic
    put32(file, 2u);         // version 2, single-part scanline
    {
        std::vector<unsigned char> ch;
        for (const char *name : {"A", "B", "G", "R"}) {
            putStr(ch, name);
            put32(ch, 2u);  // FLOAT
            ch.push_back(0);  // pLinear
            ch.push_back(0);
            ch.push_back(0);
            ch.push_back(0);
            put32(ch, 1u);  // x sampling
            put32(ch, 1u);  // y sampling
        }
        ch.push_back(0);
        attribute(file, "channels", "chlist", ch);
    }
    attribute(file, "compression", "compression", {(unsigned char)(c == ExrCompression::Zip ? 3 : 0)});
    std::vector<unsigned char> box;
    put32(box, 0u);
    put32(box, 0u);
    put32(box, width - 1u);
    put32(box, height - 1u);
    attribute(file, "dataWindow", "box2i", box);
    attribute(file, "displayWindow", "box2i", box);
    attribute(file, "lineOrder", "lineOrder", {0});
    std::vector<unsigned char> one;
    putF(one, 1.0f);
    attribute(file, "pixelAspectRatio", "float", one);
    std::vector<unsigned char> centre;
    putF(centre, 0.0f);
    putF(centre, 0.0f);
    attribute(file, "screenWindowCenter", "v2f", centre);
    attribute(file, "screenWindowWidth", "float", one);
    file.push_back(0);  // end of header

    const size_t tableAt = file.size();
    file.resize(file.size() + 8 * (size_t)chunks);
    std::vector<unsigned char> raw, pre, packed;
    for (uint32_t k = 0; k < chunks; k++) {
        const uint32_t y0 = k * linesPerChunk, y1 = std::min(height, y0 + linesPerChunk);
        raw.clear();
        for (uint32_t y = y0; y < y1; y++)
            for (int channel = 3; channel >= 0; channel--)  // A, B, G, R
                for (uint32_t x = 0; x < width; x++) putF(raw, rgba[4 * ((size_t)y * width + x) + channel]);
        const std::vector<unsigned char> *data = &raw;
        if (c == ExrCompression::Zip) {
            zipPredict(raw, pre);
            uLongf size = compressBound((uLong)pre.size());
            packed.resize(size);
            if (compress2(packed.data(), &size, pre.data(), (uLong)pre.size(), Z_DEFAULT_COMPRESSION) != Z_OK)
                return "zlib compression failed";
            packed.resize(size);
            if (packed.size() < raw.size()) data = &packed;  // else stored as is, which readers detect by size
        }
        const uint64_t at = file.size();
        for (int b = 0; b < 8; b++) file[tableAt + 8 * (size_t)k + b] = (unsigned char)(at >> (8 * b));
        put32(file, y0);
        put32(file, (uint32_t)data->size());
        file.insert(file.end(), data->begin(), data->end());
    }
    std::unique_ptr<FILE, int (*)(FILE *)> f(std::fopen(path, "wb"), &std::fclose);
    if (!f) return std::string("cannot open ") + path + " for writing";
    if (std::fwrite(file.data(), 1, file.size(), f.get()) != file.size()) return std::string("short write to ") + path;
    return "";
}

std::string writeExrFilm(const char *path, const float *rgb, uint32_t width, uint32_t height, float norm,
                         ExrCompression c) {
    if (!rgb) return "NULL film";
    std::vector<float> rgba(4 * (size_t)width * height);
    for (size_t i = 0; i < (size_t)width * height; i++) {
        rgba[4 * i + 0] = rgb[3 * i + 0] * norm;
        rgba[4 * i + 1] = rgb[3 * i + 1] * norm;
        rgba[4 * i + 2] = rgb[3 * i + 2] * norm;
        rgba[4 * i + 3] = 1.0f;
    }
    return writeExrRgba(path, rgba.data(), width, height, c);
}

}  // namespace rmdhost
