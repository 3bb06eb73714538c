// image_io.cpp -- PNG / JPEG / BMP / TGA / Radiance HDR / PGM reading and Radiance HDR writing for the command line.
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

// 8-bit pixels with n = 1 (gray), 3 (RGB) or 4 (RGBA) channels, row-major top-down, to the float image
// stbi_loadf returns with `comps` channels: gray is the integer luma of RGB (alpha ignored), RGB
// replicates gray, and every 8-bit value goes through the LDR-to-float table.
void ldr_to_image(const std::vector<uint8_t> &px, int n, int W, int H, int comps, std::vector<float> &img) {
    const float *lut = ldr_to_float_table();
    const size_t npx = static_cast<size_t>(W) * H;
    img.resize(npx * comps);
    for (size_t i = 0; i < npx; i++) {
        const uint8_t *p = &px[i * n];
        if (comps == 1) {
            img[i] = lut[n == 1 ? p[0] : luma(p[0], p[1], p[2])];
        } else {
            for (int k = 0; k < 3; k++) img[i * 3 + k] = lut[n == 1 ? p[0] : p[k]];
        }
    }
}

inline uint32_t le16(const uint8_t *p) { return uint32_t(p[0]) | (uint32_t(p[1]) << 8); }
inline uint32_t le32(const uint8_t *p) { return le16(p) | (le16(p + 2) << 16); }

// An n-bit field (n = 1..8) widened to 8 bits by repeating its bits (n = 5: v << 3 | v >> 2), as stb
// does for BMP channel masks.
inline uint8_t widen_bits(uint32_t v, int n) {
    if (n <= 0) return 0;
    if (n >= 8) return static_cast<uint8_t>(v >> (n - 8));
    uint32_t x = v << (8 - n);
    for (int k = n; k < 8; k += n) x |= x >> n;
    return static_cast<uint8_t>(x);
}

// Windows / OS2 BMP: 1, 4, 8 bits with a palette, 16/24/32 bits (BI_RGB or BI_BITFIELDS masks), bottom-up
// or (negative height) top-down, rows padded to 4 bytes.  Compressed (RLE) files are refused, as stb
// refuses them.
bool load_bmp(const std::vector<uint8_t> &f, std::vector<float> &img, int &W, int &H, int comps, std::string &err) {
    if (f.size() < 26) return err = "truncated BMP", false;
    const uint32_t data_off = le32(&f[10]), hsz = le32(&f[14]);
    if (hsz != 12 && hsz != 40 && hsz != 56 && hsz != 108 && hsz != 124) return err = "unsupported BMP header", false;
    if (f.size() < 14 + static_cast<size_t>(hsz)) return err = "truncated BMP", false;
    int w, h, bpp;
    uint32_t compress = 0;
    if (hsz == 12) {
        w = static_cast<int16_t>(le16(&f[18]));
        h = static_cast<int16_t>(le16(&f[20]));
        bpp = le16(&f[24]);
    } else {
        w = static_cast<int32_t>(le32(&f[18]));
        h = static_cast<int32_t>(le32(&f[22]));
        bpp = le16(&f[28]);
        compress = le32(&f[30]);
    }
    const bool flip = h > 0;  // stored bottom-up
    if (h < 0) h = -h;
    if (w <= 0 || h <= 0 || w > (1 << 24) || h > (1 << 24)) return err = "bad BMP size", false;
    if (compress != 0 && !(compress == 3 && (bpp == 16 || bpp == 32))) return err = "unsupported BMP compression", false;
    uint32_t mask[4] = {0, 0, 0, 0};
    if (bpp == 16) {
        mask[0] = 0x7c00;
        mask[1] = 0x03e0;
        mask[2] = 0x001f;
    } else if (bpp == 32) {
        mask[0] = 0xff0000;
        mask[1] = 0xff00;
        mask[2] = 0xff;
        mask[3] = 0xff000000u;
    }
    if (compress == 3) {
        const size_t mo = 14 + 40;  // after the 40-byte header, or inside a V4/V5 header
        if (hsz == 12 || hsz == 56 || f.size() < mo + 12) return err = "unsupported BMP bitfields", false;
        mask[0] = le32(&f[mo]);
        mask[1] = le32(&f[mo + 4]);
        mask[2] = le32(&f[mo + 8]);
    }
    std::vector<uint8_t> pal;
    if (bpp <= 8) {
        const int entry = hsz == 12 ? 3 : 4;
        const size_t pal_off = 14 + hsz;
        const size_t n = (data_off - pal_off) / entry;
        if (data_off < pal_off || n == 0 || n > 256) return err = "bad BMP palette", false;
        pal.assign(256 * 3, 0);
        for (size_t i = 0; i < n; i++)
            for (int k = 0; k < 3; k++) pal[i * 3 + k] = f[pal_off + i * entry + 2 - k];  // stored B, G, R
    } else if (bpp != 16 && bpp != 24 && bpp != 32) {
        return err = "unsupported BMP bit depth", false;
    }
    int shift[4], bits[4];
    for (int c = 0; c < 4; c++) {
        shift[c] = 0;
        bits[c] = 0;
        if (mask[c]) {
            uint32_t m = mask[c];
            while (!(m & 1u)) m >>= 1, shift[c]++;
            while (m & 1u) m >>= 1, bits[c]++;
        }
    }
    if (bpp == 16 || bpp == 32) {  // stb refuses missing colour masks and fields wider than 8 bits
        if (!mask[0] || !mask[1] || !mask[2]) return err = "bad BMP masks", false;
        for (int c = 0; c < 4; c++)
            if (bits[c] > 8) return err = "bad BMP masks", false;
    }
    const size_t stride = ((static_cast<size_t>(w) * bpp + 31) / 32) * 4;
    if (f.size() < data_off + stride * h) return err = "truncated BMP", false;
    W = w;
    H = h;
    std::vector<uint8_t> px(static_cast<size_t>(w) * h * 3);
    for (int y = 0; y < h; y++) {
        const uint8_t *row = &f[data_off + stride * (flip ? h - 1 - y : y)];
        uint8_t *dst = &px[static_cast<size_t>(y) * w * 3];
        for (int x = 0; x < w; x++, dst += 3) {
            if (bpp <= 8) {
                const int per = 8 / bpp, b = x / per, k = per - 1 - x % per;
                const int idx = (row[b] >> (k * bpp)) & ((1 << bpp) - 1);
                std::memcpy(dst, &pal[idx * 3], 3);
            } else if (bpp == 24) {
                dst[0] = row[3 * x + 2];
                dst[1] = row[3 * x + 1];
                dst[2] = row[3 * x];
            } else {
                const uint32_t v = bpp == 16 ? le16(row + 2 * x) : le32(row + 4 * x);
                for (int c = 0; c < 3; c++) dst[c] = widen_bits((v & mask[c]) >> shift[c], bits[c]);
            }
        }
    }
    ldr_to_image(px, 3, w, h, comps, img);
    return true;
}

// Truevision TGA: color-mapped (1, 9), truecolor (2, 10) and gray (3, 11) images, raw or run-length;
// 8/15/16/24/32 bits; bottom-up unless the descriptor's top-left bit is set.  15/16-bit pixels are
// 5-5-5 with each field scaled as v * 255 / 31 (stb's TGA reader).
bool load_tga(const std::vector<uint8_t> &f, std::vector<float> &img, int &W, int &H, int comps, std::string &err) {
    if (f.size() < 18) return err = "truncated TGA", false;
    const int id_len = f[0], cmap_type = f[1], type = f[2];
    const int cmap_first = le16(&f[3]), cmap_len = le16(&f[5]), cmap_bits = f[7];
    const int w = le16(&f[12]), h = le16(&f[14]), bpp = f[16], desc = f[17];
    const bool rle = type >= 9;
    const int base = rle ? type - 8 : type;
    if ((base != 1 && base != 2 && base != 3) || w <= 0 || h <= 0) return err = "unsupported TGA", false;
    if (base == 1 && (cmap_type != 1 || (bpp != 8 && bpp != 16))) return err = "unsupported TGA palette", false;
    if (base == 3 && bpp != 8 && bpp != 16) return err = "unsupported TGA gray depth", false;
    if (base == 2 && bpp != 15 && bpp != 16 && bpp != 24 && bpp != 32) return err = "unsupported TGA depth", false;
    size_t pos = 18 + id_len;
    // color map entries as RGB
    std::vector<uint8_t> cmap;
    auto color = [&](const uint8_t *p, int bits, uint8_t *rgb) {
        if (bits == 15 || bits == 16) {
            const uint32_t v = le16(p);
            rgb[0] = static_cast<uint8_t>((((v >> 10) & 31) * 255) / 31);
            rgb[1] = static_cast<uint8_t>((((v >> 5) & 31) * 255) / 31);
            rgb[2] = static_cast<uint8_t>(((v & 31) * 255) / 31);
        } else {  // 24 / 32: B, G, R (, A)
            rgb[0] = p[2];
            rgb[1] = p[1];
            rgb[2] = p[0];
        }
    };
    if (cmap_type == 1) {
        // as stb reads it: the first-entry field is a count of bytes skipped before the map, and pixel
        // indexes address the map directly (an index past its end reads entry 0)
        const int eb = (cmap_bits + 7) / 8;
        if (base == 1) pos += cmap_first;
        if (f.size() < pos + static_cast<size_t>(cmap_len) * eb) return err = "truncated TGA", false;
        if (base == 1) {
            if (cmap_len == 0 || (cmap_bits != 15 && cmap_bits != 16 && cmap_bits != 24 && cmap_bits != 32))
                return err = "unsupported TGA palette", false;
            cmap.assign(static_cast<size_t>(cmap_len) * 3, 0);
            for (int i = 0; i < cmap_len; i++) color(&f[pos + static_cast<size_t>(i) * eb], cmap_bits, &cmap[i * 3]);
        }
        pos += static_cast<size_t>(cmap_len) * eb;
    }
    const int n = base == 3 ? 1 : 3;
    const int pb = (bpp + 7) / 8;
    W = w;
    H = h;
    std::vector<uint8_t> px(static_cast<size_t>(w) * h * n);
    auto put = [&](size_t i, const uint8_t *p) -> bool {
        uint8_t *dst = &px[i * n];
        if (base == 3) {
            dst[0] = p[0];  // 16-bit gray: the low byte is the gray value (the high byte is alpha)
        } else if (base == 1) {
            int idx = bpp == 8 ? p[0] : static_cast<int>(le16(p));
            if (idx >= cmap_len) idx = 0;
            std::memcpy(dst, &cmap[static_cast<size_t>(idx) * 3], 3);
        } else {
            color(p, bpp, dst);
        }
        return true;
    };
    const size_t npx = static_cast<size_t>(w) * h;
    size_t i = 0;
    while (i < npx) {
        if (!rle) {
            if (pos + pb > f.size()) return err = "truncated TGA", false;
            if (!put(i++, &f[pos])) return err = "bad TGA color index", false;
            pos += pb;
            continue;
        }
        if (pos >= f.size()) return err = "truncated TGA", false;
        const int hdr = f[pos++], count = (hdr & 127) + 1;
        if (hdr & 128) {
            if (pos + pb > f.size()) return err = "truncated TGA", false;
            for (int k = 0; k < count && i < npx; k++)
                if (!put(i++, &f[pos])) return err = "bad TGA color index", false;
            pos += pb;
        } else {
            for (int k = 0; k < count && i < npx; k++) {
                if (pos + pb > f.size()) return err = "truncated TGA", false;
                if (!put(i++, &f[pos])) return err = "bad TGA color index", false;
                pos += pb;
            }
        }
    }
    if (!(desc & 32)) {  // bottom-up: flip rows
        const size_t rb = static_cast<size_t>(w) * n;
        std::vector<uint8_t> tmp(rb);
        for (int y = 0; y < h / 2; y++) {
            uint8_t *a = &px[y * rb], *b = &px[(h - 1 - y) * rb];
            std::memcpy(tmp.data(), a, rb);
            std::memcpy(a, b, rb);
            std::memcpy(b, tmp.data(), rb);
        }
    }
    ldr_to_image(px, n, w, h, comps, img);
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
    if (f.size() >= 2 && f[0] == 'B' && f[1] == 'M') return load_bmp(f, img, width, height, comps, err);
    if (f.size() >= 3 && f[0] == 0xff && f[1] == 0xd8 && f[2] == 0xff) {
        std::vector<uint8_t> px;
        if (!decode_jpeg(f, comps, px, width, height, err)) return false;
        ldr_to_image(px, comps, width, height, comps, img);
        return true;
    }
    // TGA has no signature: tried last, on its header's plausibility (as stb tries it last)
    if (f.size() >= 18 && (f[1] == 0 || f[1] == 1) && ((f[2] >= 1 && f[2] <= 3) || (f[2] >= 9 && f[2] <= 11)))
        return load_tga(f, img, width, height, comps, err);
    return err = "unsupported image format (PNG, JPEG, BMP, TGA, Radiance HDR and binary PGM are read)", false;
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
