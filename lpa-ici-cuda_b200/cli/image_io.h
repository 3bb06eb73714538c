// image_io.h -- the image formats the drop-in command line reads and writes.
//
// Loading returns the gray float image the reference gets from stb_image's stbi_loadf(path, .., 1)
// (src/v4_1_lpa_ici_2D_sparse_shared.cu:375):
//   * PNG (8-bit or 16-bit, gray / gray+alpha / RGB / RGBA / palette, bit depths 1-16, interlaced or
//     not): 16-bit samples keep their high byte, RGB becomes (77 R + 150 G + 29 B) >> 8, then every
//     8-bit value v becomes (float) pow(v / 255.0f, 2.2f) -- stb's LDR-to-HDR conversion;
//   * Radiance .hdr (RGBE, flat or run-length scanlines): gray = (R + G + B) * 2^(E - 136) / 3;
//   * binary PGM (P5, 8-bit), converted like 8-bit PNG gray;
//   * BMP (1/4/8-bit palettes, 16/32-bit bit fields of up to 8 bits, 24/32-bit; bottom-up or top-down; no
//     RLE) and TGA (color-mapped, truecolor 15/16/24/32-bit, gray 8/16-bit; raw or run-length), as
//     stb reads them, then converted like 8-bit PNG;
//   * baseline JPEG (1 or 3 components, any sampling factors, restart intervals; jpeg.cpp): the Y plane
//     of a YCbCr image, or the luma of an RGB-coded one, converted like 8-bit PNG.
// Writing produces a Radiance .hdr (RGBE, run-length scanlines for widths 8..32767), gray stored as
// R = G = B, as stbi_write_hdr does for one channel (src/v4_1_lpa_ici_2D_sparse_shared.cu:388, :522).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace lpaici_cli {

// Baseline JPEG to 8-bit samples with comps 1 (gray) or 3 (RGB) channels as stb_image computes them
// (jpeg.cpp); false with err on failure (progressive files included).
bool decode_jpeg(const std::vector<uint8_t> &file, int comps, std::vector<uint8_t> &px, int &width, int &height,
                 std::string &err);

// Returns false and sets err on failure.
bool load_gray(const std::string &path, std::vector<float> &img, int &width, int &height, std::string &err);
// comps 1: as load_gray; comps 3: interleaved R, G, B as stbi_loadf(path, .., 3) returns them (gray
// files replicated, alpha dropped, 16-bit samples' high bytes, HDR mantissas times 2^(E - 136)).
bool load_image(const std::string &path, int comps, std::vector<float> &img, int &width, int &height,
                std::string &err);
// comps 1 (gray, stored R = G = B) or 3 (interleaved RGB), RGBE as stbi_write_hdr encodes it.
bool write_hdr(const std::string &path, const float *img, int width, int height, int comps = 1);

// The 256 values of stb's 8-bit to float conversion (pow(v/255, 2.2)).
const float *ldr_to_float_table();

}  // namespace lpaici_cli
