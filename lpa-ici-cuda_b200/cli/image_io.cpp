// image_io.cpp -- PNG / Radiance HDR / PGM reading and Radiance HDR writing for the command line.
// Conversions follow what stb_image (v2.30) and stb_image_write (v1.16), the reference's vendored
// image libraries, do on the same files; the code is this project's own.
#include "image_io.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>

namespace lpaici_cli {

namespace {

// 8-bit RGB to gray, the integer luma of stb_image (stb_image.h:1746).
inline uint8_t luma(int r, int g, int b) { return static_cast<uint8_t>(((r * 77) + (g * 150) + (29 * b)) >> 8); }
inline uint16_t luma16(int r, int g, int b) {
    return static_cast<uint16_t>(((r * 77) + (g * 150) + (29 * b)) >> 8);
}

bool read_file(const std::string &path, std::vector<uint8_t> &buf) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

uint32_t be32(const uint8_t *p) { return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    if (pb <= pc) return b;
    return c;
}

// Reverses the PNG row filters of a (sub-)image of w x h pixels in place; returns the raw rows.
bool unfilter(const uint8_t *src, size_t avail, int w, int h, int bits_pp, std::vector<uint8_t> &rows,
              size_t &consumed) {
    const size_t stride = (static_cast<size_t>(w) * bits_pp + 7) / 8;
    const int bpp = bits_pp >= 8 ? bits_pp / 8 : 1;
    rows.assign(stride * h, 0);
    consumed = (stride + 1) * h;
    if (w == 0 || h == 0) {
        consumed = 0;
        return true;
    }
    if (avail < consumed) return false;
    for (int y = 0; y < h; y++) {
        const uint8_t ft = src[y * (stride + 1)];
        const uint8_t *in = src + y * (stride + 1) + 1;
        uint8_t *out = rows.data() + y * stride;
        const uint8_t *prev = y ? out - stride : nullptr;
        for (size_t i = 0; i < stride; i++) {
            const int a = i >= static_cast<size_t>(bpp) ? out[i - bpp] : 0;
            const int b = prev ? prev[i] : 0;
            const int c = (prev && i >= static_cast<size_t>(bpp)) ? prev[i - bpp] : 0;
            int v = in[i];
            switch (ft) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) >> 1; break;
                case 4: v += paeth(a, b, c); break;
                default: return false;
            }
            out[i] = static_cast<uint8_t>(v);
        }
    }
    return true;
}

// One PNG sample (channel ch of pixel x in a raw row) at the file's bit depth.
inline int sample(const uint8_t *row, int x, int ch, int channels, int depth) {
    if (depth == 8) return row[x * channels + ch];
    if (depth == 16) {
        const uint8_t *p = row + 2 * (x * channels + ch);
        return (p[0] << 8) | p[1];
    }
    const int idx = x * channels + ch, per = 8 / depth;  // sub-byte depths only for 1-channel types
    const int shift = 8 - depth * (idx % per + 1);
    return (row[idx / per] >> shift) & ((1 << depth) - 1);
}

bool load_png(const std::vector<uint8_t> &f, std::vector<float> &img, int &W, int &H, int comps, std::string &err) {
    if (f.size() < 8 + 25) return err = "truncated PNG", false;
    size_t pos = 8;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte;
    bool have_ihdr = false;
    while (pos + 12 <= f.size()) {
        const uint32_t len = be32(&f[pos]);
        if (pos + 12 + static_cast<size_t>(len) > f.size()) return err = "corrupt PNG chunk", false;
        const uint8_t *type = &f[pos + 4], *data = &f[pos + 8];
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) return err = "bad IHDR", false;
            W = static_cast<int>(be32(data));
            H = static_cast<int>(be32(data + 4));
            depth = data[8];
            ctype = data[9];
            interlace = data[12];
            have_ihdr = true;
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(data, data + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            break;
        }
        pos += 12 + len;
    }
    if (!have_ihdr || W <= 0 || H <= 0 || W > (1 << 24) || H > (1 << 24)) return err = "bad PNG header", false;
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: return err = "unsupported PNG color type", false;
    }
    const bool ok_depth = (ctype == 0 && (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) ||
                          (ctype == 3 && (depth == 1 || depth == 2 || depth == 4 || depth == 8)) ||
                          ((ctype == 2 || ctype == 4 || ctype == 6) && (depth == 8 || depth == 16));
    if (!ok_depth) return err = "unsupported PNG bit depth", false;
    if (ctype == 3 && plte.size() < 3) return err = "PNG palette missing", false;
    const int bits_pp = channels * depth;

    // inflate the concatenated IDAT stream
    size_t raw_cap = 0;
    if (interlace == 0) {
        raw_cap = ((static_cast<size_t>(W) * bits_pp + 7) / 8 + 1) * H;
    } else {
        for (int p = 0; p < 7; p++) {
            static const int xo[7] = {0, 4, 0, 2, 0, 1, 0}, yo[7] = {0, 0, 4, 0, 2, 0, 1};
            static const int xs[7] = {8, 8, 4, 4, 2, 2, 1}, ys[7] = {8, 8, 8, 4, 4, 2, 2};
            const size_t pw = (W - xo[p] + xs[p] - 1) / xs[p], ph = (H - yo[p] + ys[p] - 1) / ys[p];
            if (pw && ph) raw_cap += ((pw * bits_pp + 7) / 8 + 1) * ph;
        }
    }
    std::vector<uint8_t> raw(raw_cap + 1);
    uLongf raw_len = static_cast<uLongf>(raw.size());
    if (uncompress(raw.data(), &raw_len, idat.data(), static_cast<uLong>(idat.size())) != Z_OK)
        return err = "corrupt PNG data", false;

    // 8-bit samples per pixel: gray (comps 1; 16-bit samples: gray conversion at 16 bits, then the
    // high byte) or R, G, B (comps 3; gray replicated, alpha dropped, 16-bit samples' high bytes)
    std::vector<uint8_t> gray(static_cast<size_t>(W) * H * comps);
    static const int scale[9] = {0, 0xff, 0x55, 0, 0x11, 0, 0, 0, 0x01};
    auto put_row = [&](const uint8_t *row, int n, int y, int x0, int dx) {
        for (int i = 0; i < n; i++) {
            int rgb[3] = {0, 0, 0}, g = 0;
            bool color = false;
            if (ctype == 3) {
                const int idx = sample(row, i, 0, 1, depth);
                if (3 * idx + 2 < static_cast<int>(plte.size()))
                    for (int k = 0; k < 3; k++) rgb[k] = plte[3 * idx + k];
                color = true;
            } else if (depth == 16) {
                if (channels >= 3) {
                    for (int k = 0; k < 3; k++) rgb[k] = sample(row, i, k, channels, 16);
                    if (comps == 1) {
                        g = (luma16(rgb[0], rgb[1], rgb[2]) >> 8) & 0xff;
                    } else {
                        for (int k = 0; k < 3; k++) rgb[k] >>= 8;
                        color = true;
                    }
                } else {
                    g = (sample(row, i, 0, channels, 16) >> 8) & 0xff;
                }
            } else if (channels >= 3) {
                for (int k = 0; k < 3; k++) rgb[k] = sample(row, i, k, channels, 8);
                color = true;
            } else {
                const int v = sample(row, i, 0, channels, depth);
                g = depth < 8 ? v * scale[depth] : v;
            }
            uint8_t *dst = &gray[(static_cast<size_t>(y) * W + x0 + static_cast<size_t>(i) * dx) * comps];
            if (comps == 1) {
                dst[0] = static_cast<uint8_t>(color ? luma(rgb[0], rgb[1], rgb[2]) : g);
            } else {
                for (int k = 0; k < 3; k++) dst[k] = static_cast<uint8_t>(color ? rgb[k] : g);
            }
        }
    };
    if (interlace == 0) {
        std::vector<uint8_t> rows;
        size_t used = 0;
        if (!unfilter(raw.data(), raw_len, W, H, bits_pp, rows, used)) return err = "corrupt PNG rows", false;
        const size_t stride = (static_cast<size_t>(W) * bits_pp + 7) / 8;
        for (int y = 0; y < H; y++) put_row(rows.data() + y * stride, W, y, 0, 1);
    } else {
        static const int xo[7] = {0, 4, 0, 2, 0, 1, 0}, yo[7] = {0, 0, 4, 0, 2, 0, 1};
        static const int xs[7] = {8, 8, 4, 4, 2, 2, 1}, ys[7] = {8, 8, 8, 4, 4, 2, 2};
        size_t off = 0;
        for (int p = 0; p < 7; p++) {
            const int pw = (W - xo[p] + xs[p] - 1) / xs[p], ph = (H - yo[p] + ys[p] - 1) / ys[p];
            if (pw <= 0 || ph <= 0) continue;
            std::vector<uint8_t> rows;
            size_t used = 0;
            if (!unfilter(raw.data() + off, raw_len - off, pw, ph, bits_pp, rows, used))
                return err = "corrupt PNG rows", false;
            off += used;
            const size_t stride = (static_cast<size_t>(pw) * bits_pp + 7) / 8;
            for (int y = 0; y < ph; y++) put_row(rows.data() + y * stride, pw, yo[p] + y * ys[p], xo[p], xs[p]);
        }
    }
    const float *lut = ldr_to_float_table();
    img.resize(gray.size());
    for (size_t i = 0; i < gray.size(); i++) img[i] = lut[gray[i]];
    return true;
}

bool load_pgm(const std::vector<uint8_t> &f, std::vector<float> &img, int &W, int &H, int comps, std::string &err) {
    size_t pos = 2;
    int vals[3] = {0, 0, 0}, n = 0;
    while (n < 3 && pos < f.size()) {
        while (pos < f.size() && (std::isspace(f[pos]) || f[pos] == '#')) {
            if (f[pos] == '#')
                while (pos < f.size() && f[pos] != '\n') pos++;
            else
                pos++;
        }
        int v = 0, digits = 0;
        while (pos < f.size() && f[pos] >= '0' && f[pos] <= '9') v = v * 10 + (f[pos++] - '0'), digits++;
        if (!digits) return err = "bad PGM header", false;
        vals[n++] = v;
    }
    pos++;  // single whitespace after maxval
    W = vals[0];
    H = vals[1];
    if (n < 3 || W <= 0 || H <= 0 || vals[2] != 255) return err = "unsupported PGM (8-bit P5 only)", false;
    if (f.size() < pos + static_cast<size_t>(W) * H) return err = "truncated PGM", false;
    const float *lut = ldr_to_float_table();
    img.resize(static_cast<size_t>(W) * H * comps);
    for (size_t i = 0; i < img.size(); i++) img[i] = lut[f[pos + i / comps]];
    return true;
}

// RGBE pixel to gray: (R + G + B) * 2^(E - 136) / 3 in float, 0 when E == 0; to RGB: each
// mantissa byte times 2^(E - 136).
inline float rgbe_gray(const uint8_t *p) {
    if (p[3] == 0) return 0.0f;
    const float f1 = static_cast<float>(std::ldexp(1.0f, p[3] - static_cast<int>(128 + 8)));
    return (p[0] + p[1] + p[2]) * f1 / 3;
}
inline void rgbe_decode(const uint8_t *p, int comps, float *out) {
    if (comps == 1) {
        out[0] = rgbe_gray(p);
        return;
    }
    const float f1 = p[3] ? static_cast<float>(std::ldexp(1.0f, p[3] - static_cast<int>(128 + 8))) : 0.0f;
    for (int k = 0; k < 3; k++) out[k] = p[3] ? p[k] * f1 : 0.0f;
}

bool load_hdr(const std::vector<uint8_t> &f, std::vector<float> &img, int &W, int &H, int comps, std::string &err) {
    size_t pos = 0;
    auto line = [&]() {
        std::string s;
        while (pos < f.size() && f[pos] != '\n') s += static_cast<char>(f[pos++]);
        if (pos < f.size()) pos++;
        return s;
    };
    const std::string magic = line();
    if (magic != "#?RADIANCE" && magic != "#?RGBE") return err = "not a Radiance file", false;
    bool fmt = false;
    for (;;) {
        if (pos >= f.size()) return err = "truncated HDR header", false;
        const std::string s = line();
        if (s.empty()) break;
        if (s == "FORMAT=32-bit_rle_rgbe") fmt = true;
    }
    if (!fmt) return err = "unsupported HDR format", false;
    const std::string dims = line();
    if (std::sscanf(dims.c_str(), "-Y %d +X %d", &H, &W) != 2 || W <= 0 || H <= 0 || W > (1 << 24) || H > (1 << 24))
        return err = "unsupported HDR orientation or size", false;
    img.assign(static_cast<size_t>(W) * H * comps, 0.0f);
    auto flat = [&](size_t from_px) {
        for (size_t i = from_px; i < static_cast<size_t>(W) * H; i++) {
            if (pos + 4 > f.size()) return false;
            rgbe_decode(&f[pos], comps, &img[i * comps]);
            pos += 4;
        }
        return true;
    };
    if (W < 8 || W >= 32768) {
        if (!flat(0)) return err = "truncated HDR data", false;
        return true;
    }
    std::vector<uint8_t> scan(static_cast<size_t>(W) * 4);
    for (int y = 0; y < H; y++) {
        if (pos + 4 > f.size()) return err = "truncated HDR data", false;
        const uint8_t *h = &f[pos];
        if (h[0] != 2 || h[1] != 2 || (h[2] & 0x80)) {
            if (y != 0) return err = "mixed flat and run-length HDR scanlines", false;
            if (!flat(0)) return err = "truncated HDR data", false;  // flat file: h is the first pixel
            return true;
        }
        if (((h[2] << 8) | h[3]) != W) return err = "bad HDR scanline width", false;
        pos += 4;
        for (int k = 0; k < 4; k++) {
            int x = 0;
            while (x < W) {
                if (pos >= f.size()) return err = "truncated HDR data", false;
                int count = f[pos++];
                if (count > 128) {
                    count -= 128;
                    if (count > W - x || pos >= f.size()) return err = "bad HDR run", false;
                    const uint8_t v = f[pos++];
                    for (int i = 0; i < count; i++) scan[4 * (x++) + k] = v;
                } else {
                    if (count == 0 || count > W - x || pos + count > f.size()) return err = "bad HDR dump", false;
                    for (int i = 0; i < count; i++) scan[4 * (x++) + k] = f[pos++];
                }
            }
        }
        for (int x = 0; x < W; x++) rgbe_decode(&scan[4 * x], comps, &img[(static_cast<size_t>(y) * W + x) * comps]);
    }
    return true;
}

// Linear R, G, B to RGBE: with m = max(R, G, B), every channel's mantissa is c * (frexp(m) * 256 / m)
// truncated to 8 bits, the exponent frexp's + 128; all zero when m < 1e-32.  Gray is R = G = B.
inline void rgb_rgbe(const float *c, uint8_t *out) {
    const float m = std::max(std::max(c[0], c[1]), c[2]);
    if (m < 1e-32f) {
        out[0] = out[1] = out[2] = out[3] = 0;
        return;
    }
    int e = 0;
    const float normalize = static_cast<float>(std::frexp(m, &e)) * 256.0f / m;
    for (int k = 0; k < 3; k++) out[k] = static_cast<uint8_t>(c[k] * normalize);
    out[3] = static_cast<uint8_t>(e + 128);
}
inline void pixel_rgbe(const float *px, int comps, uint8_t *out) {
    const float c[3] = {px[0], px[comps == 1 ? 0 : 1], px[comps == 1 ? 0 : 2]};
    rgb_rgbe(c, out);
}

// Radiance run-length coding of one component line: runs of >= 3 equal bytes as (128 + n, byte),
// n <= 127; everything else as literal blocks (n, bytes...), n <= 128.
void rle_component(const uint8_t *c, int n, std::vector<uint8_t> &out) {
    int x = 0;
    while (x < n) {
        int r = x;  // start of the next run of three equal bytes
        while (r + 2 < n && !(c[r] == c[r + 1] && c[r] == c[r + 2])) r++;
        if (r + 2 >= n) r = n;
        while (x < r) {
            const int len = std::min(r - x, 128);
            out.push_back(static_cast<uint8_t>(len));
            out.insert(out.end(), c + x, c + x + len);
            x += len;
        }
        if (r < n) {
            int e = r;
            while (e < n && c[e] == c[r]) e++;
            while (x < e) {
                const int len = std::min(e - x, 127);
                out.push_back(static_cast<uint8_t>(128 + len));
                out.push_back(c[x]);
                x += len;
            }
        }
    }
}

}  // namespace

const float *ldr_to_float_table() {
    static float table[256];
    static bool init = false;
    if (!init) {
        for (int v = 0; v < 256; v++)  // equal to stb's result on all 256 levels (checked by the tests)
            table[v] = static_cast<float>(std::pow(static_cast<double>(v / 255.0f), static_cast<double>(2.2f)) * 1.0);
        init = true;
    }
    return table;
}

bool load_image(const std::string &path, int comps, std::vector<float> &img, int &width, int &height,
                std::string &err) {
    if (comps != 1 && comps != 3) return err = "1 or 3 channels", false;
    std::vector<uint8_t> f;
    if (!read_file(path, f)) return err = "cannot open file", false;
    static const uint8_t png_sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (f.size() >= 8 && !std::memcmp(f.data(), png_sig, 8)) return load_png(f, img, width, height, comps, err);
    if (f.size() >= 2 && f[0] == '#' && f[1] == '?') return load_hdr(f, img, width, height, comps, err);
    if (f.size() >= 2 && f[0] == 'P' && f[1] == '5') return load_pgm(f, img, width, height, comps, err);
    return err = "unsupported image format (PNG, Radiance HDR and binary PGM are read)", false;
}

bool load_gray(const std::string &path, std::vector<float> &img, int &width, int &height, std::string &err) {
    return load_image(path, 1, img, width, height, err);
}

bool write_hdr(const std::string &path, const float *img, int width, int height, int comps) {
    if (width <= 0 || height <= 0 || !img || (comps != 1 && comps != 3)) return false;
    std::vector<uint8_t> out;
    const std::string head = "#?RADIANCE\n# Written by lpaici\nFORMAT=32-bit_rle_rgbe\n"
                             "EXPOSURE=          1.0000000000000\n\n-Y " +
                             std::to_string(height) + " +X " + std::to_string(width) + "\n";
    out.insert(out.end(), head.begin(), head.end());
    std::vector<uint8_t> comp(static_cast<size_t>(width) * 4);
    for (int y = 0; y < height; y++) {
        const float *row = img + static_cast<size_t>(y) * width * comps;
        if (width < 8 || width >= 32768) {
            for (int x = 0; x < width; x++) {
                uint8_t p[4];
                pixel_rgbe(row + static_cast<size_t>(x) * comps, comps, p);
                out.insert(out.end(), p, p + 4);
            }
            continue;
        }
        for (int x = 0; x < width; x++) {
            uint8_t p[4];
            pixel_rgbe(row + static_cast<size_t>(x) * comps, comps, p);
            for (int k = 0; k < 4; k++) comp[static_cast<size_t>(k) * width + x] = p[k];
        }
        out.push_back(2);
        out.push_back(2);
        out.push_back(static_cast<uint8_t>((width >> 8) & 0xff));
        out.push_back(static_cast<uint8_t>(width & 0xff));
        for (int k = 0; k < 4; k++) rle_component(&comp[static_cast<size_t>(k) * width], width, out);
    }
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    f.write(reinterpret_cast<const char *>(out.data()), static_cast<std::streamsize>(out.size()));
    return static_cast<bool>(f);
}

}  // namespace lpaici_cli

// C entry points of lib/liblpaici_io.so (the command line's image I/O, for other callers and tests).
extern "C" {

// Loads a gray float image; *out is malloc'd (free with lpaici_io_free).  Returns 0 or -1.
__attribute__((visibility("default"))) int lpaici_io_load_gray(const char *path, float **out, int *width,
                                                               int *height) {
    std::vector<float> img;
    std::string err;
    int w = 0, h = 0;
    if (!path || !out || !lpaici_cli::load_gray(path, img, w, h, err)) return -1;
    *out = static_cast<float *>(std::malloc(sizeof(float) * img.size()));
    if (!*out) return -1;
    std::memcpy(*out, img.data(), sizeof(float) * img.size());
    *width = w;
    *height = h;
    return 0;
}

__attribute__((visibility("default"))) void lpaici_io_free(void *p) { std::free(p); }

// Writes a one-channel float image as Radiance .hdr.  Returns 0 or -1.
__attribute__((visibility("default"))) int lpaici_io_write_hdr(const char *path, const float *img, int width,
                                                               int height) {
    return path && lpaici_cli::write_hdr(path, img, width, height, 1) ? 0 : -1;
}

// Loads an RGB float image (width x height x 3, interleaved), as stbi_loadf(path, .., 3) returns it;
// *out is malloc'd (free with lpaici_io_free).  Returns 0 or -1.
__attribute__((visibility("default"))) int lpaici_io_load_rgb(const char *path, float **out, int *width, int *height) {
    std::vector<float> img;
    std::string err;
    int w = 0, h = 0;
    if (!path || !out || !lpaici_cli::load_image(path, 3, img, w, h, err)) return -1;
    *out = static_cast<float *>(std::malloc(sizeof(float) * img.size()));
    if (!*out) return -1;
    std::memcpy(*out, img.data(), sizeof(float) * img.size());
    *width = w;
    *height = h;
    return 0;
}

// Writes an interleaved RGB float image as Radiance .hdr.  Returns 0 or -1.
__attribute__((visibility("default"))) int lpaici_io_write_hdr_rgb(const char *path, const float *img, int width,
                                                                   int height) {
    return path && lpaici_cli::write_hdr(path, img, width, height, 3) ? 0 : -1;
}
}
