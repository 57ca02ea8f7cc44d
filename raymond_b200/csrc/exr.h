// OpenEXR writer of the film (exr.cpp).
#pragma once
#include <cstdint>
#include <string>

namespace rmdhost {

enum class ExrCompression : uint32_t { Auto = 0, None = 1, Zip = 2 };

// rgba: width x height x 4 floats, row-major from the top-left pixel.
// Returns an error message, empty on success.
std::string writeExrRgba(const char *path, const float *rgba, uint32_t width, uint32_t height, ExrCompression c);
// rgb: width x height x 3 floats (a raw film); colours times norm, alpha 1.
std::string writeExrFilm(const char *path, const float *rgb, uint32_t width, uint32_t height, float norm,
                         ExrCompression c);

}  // namespace rmdhost
