// rt_image.h - image codecs without an image library: PNG decoding and
// encoding (rt_png.cpp), baseline JPEG decoding (rt_jpeg.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace rti {
// A zlib stream (RFC 1950 / 1951) of at most `expected` bytes.
bool zlib_inflate(const uint8_t* src, size_t n, std::vector<uint8_t>& out, size_t expected, std::string& err);
// PNG file bytes -> RGBA8, row 0 = bottom (stbi_load + vertical flip).
// Colour types grey, RGB, palette, grey+alpha, RGBA; bit depths 1-16; not interlaced.
bool read_png(const std::string& file, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err);
// RGBA8 frame (row 0 = bottom, as DownloadPixels) -> PNG file.
bool write_png(const std::string& path, const uint32_t* rgba8, int w, int h, std::string& err);
// JPEG file bytes -> RGBA8, row 0 = bottom.  Baseline / extended sequential
// Huffman-coded, 8-bit, grey or YCbCr, one interleaved scan.
bool read_jpeg(const std::string& file, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err);
}  // namespace rti
