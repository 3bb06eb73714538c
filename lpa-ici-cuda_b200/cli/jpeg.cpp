// jpeg.cpp -- baseline JPEG decoding for the command line, with the arithmetic of stb_image (v2.30), the
// reference's loader (stbi_loadf, src/v4_1_lpa_ici_2D_sparse_shared.cu:375), so the 8-bit samples it
// produces are the ones stb produces:
//   * Huffman-coded sequential DCT (SOF0/SOF1), 8-bit samples, 1 or 3 components, any sampling factors,
//     restart intervals; coefficients dequantised into 16-bit integers;
//   * the separable 8x8 integer inverse DCT of the IJG "islow" method (Loeffler-Ligtenberg-Moschytz
//     flow graph) with 12-bit fixed-point constants, 2 extra bits kept between the column and the row
//     pass, +128 level shift, clamped to 0..255;
//   * chroma upsampling by stb's filters: 3:1 triangle weights horizontally and/or vertically ("fancy"),
//     nearest for other factors; YCbCr to RGB in 20-bit fixed point (the Cb term of green truncated to
//     16 fraction bits, as stb's SIMD path computes it);
//   * gray output of a YCbCr image is its Y plane; of an RGB-coded image, the integer luma of R, G, B.
// Progressive and arithmetic-coded files are refused.  The code is this project's own.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace lpaici_cli {

namespace {

const uint8_t kZigzag[64 + 16] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                  12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                  35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                  58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63,
                                  // runs past coefficient 63 in a corrupt stream land here, harmlessly
                                  63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63};

struct Huffman {
    // canonical code tables: for code length l (1..16), codes [first[l], first[l] + count[l]) map to
    // symbols starting at index base[l]
    int first[17], count[17], base[17];
    uint8_t sym[256];
    bool ok = false;
};

struct Component {
    int id, h, v, tq, td, ta;
    int bw, bh;                 // blocks across / down (whole MCUs)
    std::vector<uint8_t> data;  // decoded samples, bw * 8 x bh * 8
    int dc_pred = 0;
};

struct Decoder {
    const uint8_t *p, *end;
    uint16_t q[4][64];
    bool q_ok[4] = {false, false, false, false};
    Huffman hdc[4], hac[4];
    std::vector<Component> comp;
    int W = 0, H = 0, hmax = 1, vmax = 1, restart = 0;
    bool jfif = false;
    int adobe_transform = -1;
    std::string err;
    // entropy-coded bit reader
    uint32_t bits = 0;
    int nbits = 0;
    bool marker_hit = false;

    bool fail(const char *m) {
        err = m;
        return false;
    }
    int u8() { return p < end ? *p++ : 0; }
    int u16() {
        const int a = u8();
        return (a << 8) | u8();
    }

    void fill() {
        while (nbits <= 24) {
            int c = 0;
            if (!marker_hit && p < end) {
                c = *p;
                if (c == 0xff) {
                    const int n = p + 1 < end ? p[1] : 0xd9;
                    if (n == 0) {
                        p += 2;  // stuffed zero byte
                    } else {
                        marker_hit = true;  // a marker ends the segment: feed zeros
                        c = 0;
                    }
                } else {
                    p++;
                }
            }
            bits |= static_cast<uint32_t>(c) << (24 - nbits);
            nbits += 8;
        }
    }
    int getbit() {
        if (nbits < 1) fill();
        const int b = static_cast<int>(bits >> 31);
        bits <<= 1;
        nbits--;
        return b;
    }
    int getbits(int n) {
        if (n == 0) return 0;
        if (nbits < n) fill();
        const int v = static_cast<int>(bits >> (32 - n));
        bits <<= n;
        nbits -= n;
        return v;
    }
    // the value of an n-bit magnitude category (JPEG's EXTEND)
    int receive_extend(int n) {
        if (n == 0) return 0;
        const int v = getbits(n);
        return v < (1 << (n - 1)) ? v - (1 << n) + 1 : v;
    }
    int decode(const Huffman &h) {
        int code = 0;
        for (int l = 1; l <= 16; l++) {
            code = (code << 1) | getbit();
            if (code >= h.first[l] && code - h.first[l] < h.count[l]) return h.sym[h.base[l] + code - h.first[l]];
        }
        return -1;
    }

    bool read_dht(int len) {
        while (len > 0) {
            const int tc_th = u8();
            const int tc = tc_th >> 4, th = tc_th & 15;
            if (tc > 1 || th > 3) return fail("bad JPEG Huffman table");
            Huffman &h = tc == 0 ? hdc[th] : hac[th];
            int total = 0, code = 0;
            for (int l = 1; l <= 16; l++) {
                h.count[l] = u8();
                h.base[l] = total;
                h.first[l] = code;
                total += h.count[l];
                code = (code + h.count[l]) << 1;
            }
            if (total > 256) return fail("bad JPEG Huffman table");
            for (int i = 0; i < total; i++) h.sym[i] = static_cast<uint8_t>(u8());
            h.ok = true;
            len -= 17 + total;
        }
        return len == 0 || fail("bad JPEG Huffman table length");
    }
    bool read_dqt(int len) {
        while (len > 0) {
            const int pq_tq = u8();
            const int pq = pq_tq >> 4, tq = pq_tq & 15;
            if (pq > 1 || tq > 3) return fail("bad JPEG quantisation table");
            for (int i = 0; i < 64; i++) q[tq][kZigzag[i]] = static_cast<uint16_t>(pq ? u16() : u8());
            q_ok[tq] = true;
            len -= 65 + 64 * pq;
        }
        return len == 0 || fail("bad JPEG quantisation table length");
    }
    bool read_sof(int len) {
        if (u8() != 8) return fail("only 8-bit JPEG samples are read");
        H = u16();
        W = u16();
        const int n = u8();
        if (W <= 0 || H <= 0) return fail("bad JPEG size (a DNL marker is not supported)");
        if (n != 1 && n != 3) return fail("only 1- and 3-component JPEG images are read");
        if (len != 6 + 3 * n) return fail("bad JPEG frame header");
        comp.resize(n);
        for (auto &c : comp) {
            c.id = u8();
            const int hv = u8();
            c.h = hv >> 4;
            c.v = hv & 15;
            c.tq = u8();
            if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) return fail("bad JPEG component");
            hmax = std::max(hmax, c.h);
            vmax = std::max(vmax, c.v);
        }
        const int mcux = (W + 8 * hmax - 1) / (8 * hmax), mcuy = (H + 8 * vmax - 1) / (8 * vmax);
        for (auto &c : comp) {
            c.bw = mcux * c.h;
            c.bh = mcuy * c.v;
            c.data.assign(static_cast<size_t>(c.bw) * 8 * c.bh * 8, 0);
        }
        return true;
    }

    bool block(Component &c, int16_t blk[64]) {
        std::memset(blk, 0, 64 * sizeof(int16_t));
        const Huffman &dc = hdc[c.td], &ac = hac[c.ta];
        if (!dc.ok || !ac.ok) return fail("missing JPEG Huffman table");
        const int t = decode(dc);
        if (t < 0 || t > 15) return fail("bad JPEG Huffman code");
        c.dc_pred += receive_extend(t);
        const uint16_t *qt = q[c.tq];
        blk[0] = static_cast<int16_t>(c.dc_pred * qt[0]);
        for (int k = 1; k < 64;) {
            const int rs = decode(ac);
            if (rs < 0) return fail("bad JPEG Huffman code");
            const int r = rs >> 4, s = rs & 15;
            if (s == 0) {
                if (r != 15) break;  // end of block
                k += 16;
                continue;
            }
            k += r;
            const int z = kZigzag[k];
            blk[z] = static_cast<int16_t>(receive_extend(s) * qt[z]);
            k++;
        }
        return true;
    }

    bool read_sos() {
        const int ns = u8();
        if (ns < 1 || ns > static_cast<int>(comp.size())) return fail("bad JPEG scan header");
        std::vector<int> sc(ns);
        for (int i = 0; i < ns; i++) {
            const int id = u8(), t = u8();
            int k = -1;
            for (size_t j = 0; j < comp.size(); j++)
                if (comp[j].id == id) k = static_cast<int>(j);
            if (k < 0) return fail("bad JPEG scan component");
            comp[k].td = t >> 4;
            comp[k].ta = t & 15;
            if (comp[k].td > 3 || comp[k].ta > 3) return fail("bad JPEG scan table");
            sc[i] = k;
        }
        const int ss = u8(), se = u8(), ahal = u8();
        if (ss != 0 || se != 63 || ahal != 0) return fail("bad JPEG scan (sequential)");
        for (const int k : sc)
            if (!q_ok[comp[k].tq]) return fail("missing JPEG quantisation table");
        bits = 0;
        nbits = 0;
        marker_hit = false;
        for (auto &c : comp) c.dc_pred = 0;
        int16_t blk[64];
        int todo = restart ? restart : 0x7fffffff;
        auto restart_marker = [&]() -> bool {
            // realign to the byte stream, expect RSTn, reset the predictors
            bits = 0;
            nbits = 0;
            marker_hit = false;
            if (p + 1 < end && p[0] == 0xff && p[1] >= 0xd0 && p[1] <= 0xd7) {
                p += 2;
            }
            for (auto &c : comp) c.dc_pred = 0;
            todo = restart;
            return true;
        };
        if (ns == 1) {
            // non-interleaved: the component's own blocks covering the image, in raster order
            Component &c = comp[sc[0]];
            const int cw = (W * c.h + hmax - 1) / hmax, ch = (H * c.v + vmax - 1) / vmax;
            const int nbx = (cw + 7) / 8, nby = (ch + 7) / 8;
            for (int by = 0; by < nby; by++)
                for (int bx = 0; bx < nbx; bx++) {
                    if (!block(c, blk)) return false;
                    idct(blk, &c.data[static_cast<size_t>(by) * 8 * c.bw * 8 + bx * 8], c.bw * 8);
                    if (--todo <= 0 && !(by == nby - 1 && bx == nbx - 1)) restart_marker();
                }
        } else {
            const int mcux = (W + 8 * hmax - 1) / (8 * hmax), mcuy = (H + 8 * vmax - 1) / (8 * vmax);
            for (int my = 0; my < mcuy; my++)
                for (int mx = 0; mx < mcux; mx++) {
                    for (const int k : sc) {
                        Component &c = comp[k];
                        for (int y = 0; y < c.v; y++)
                            for (int x = 0; x < c.h; x++) {
                                if (!block(c, blk)) return false;
                                const int bx = mx * c.h + x, by = my * c.v + y;
                                idct(blk, &c.data[static_cast<size_t>(by) * 8 * c.bw * 8 + bx * 8], c.bw * 8);
                            }
                    }
                    if (--todo <= 0 && !(my == mcuy - 1 && mx == mcux - 1)) restart_marker();
                }
        }
        // skip to the next marker
        while (p + 1 < end && !(p[0] == 0xff && p[1] != 0 && !(p[1] >= 0xd0 && p[1] <= 0xd7))) p++;
        return true;
    }

    // 8x8 inverse DCT, column pass then row pass, 12-bit constants (see the file comment)
    static inline uint8_t clamp255(int v) { return static_cast<uint8_t>(v < 0 ? 0 : (v > 255 ? 255 : v)); }
    static inline int fix(double x) { return static_cast<int>(x * 4096 + 0.5); }
    static inline void even_odd(int s0, int s1, int s2, int s3, int s4, int s5, int s6, int s7, int ev[4], int od[4]) {
        static const int c_05411961 = fix(0.5411961f), c_m1847759065 = fix(-1.847759065f), c_0765366865 = fix(0.765366865f),
                         c_1175875602 = fix(1.175875602f), c_0298631336 = fix(0.298631336f),
                         c_2053119869 = fix(2.053119869f), c_3072711026 = fix(3.072711026f),
                         c_1501321110 = fix(1.501321110f), c_m0899976223 = fix(-0.899976223f),
                         c_m2562915447 = fix(-2.562915447f), c_m1961570560 = fix(-1.961570560f),
                         c_m0390180644 = fix(-0.390180644f);
        // even part: inputs 0, 2, 4, 6
        const int z1 = (s2 + s6) * c_05411961;
        const int e2 = z1 + s6 * c_m1847759065, e3 = z1 + s2 * c_0765366865;
        const int e0 = (s0 + s4) * 4096, e1 = (s0 - s4) * 4096;
        ev[0] = e0 + e3;
        ev[3] = e0 - e3;
        ev[1] = e1 + e2;
        ev[2] = e1 - e2;
        // odd part: inputs 7, 5, 3, 1
        const int q3 = s7 + s3, q4 = s5 + s1, q1 = s7 + s1, q2 = s5 + s3;
        const int z5 = (q3 + q4) * c_1175875602;
        int o0 = s7 * c_0298631336, o1 = s5 * c_2053119869, o2 = s3 * c_3072711026, o3 = s1 * c_1501321110;
        const int r1 = z5 + q1 * c_m0899976223, r2 = z5 + q2 * c_m2562915447;
        const int r3 = q3 * c_m1961570560, r4 = q4 * c_m0390180644;
        o3 += r1 + r4;
        o2 += r2 + r3;
        o1 += r2 + r4;
        o0 += r1 + r3;
        od[0] = o3;  // pairs with ev[0]
        od[1] = o2;  // ev[1]
        od[2] = o1;  // ev[2]
        od[3] = o0;  // ev[3]
    }
    static void idct(const int16_t in[64], uint8_t *out, int stride) {
        int tmp[64];
        for (int c = 0; c < 8; c++) {
            const int16_t *d = in + c;
            if (!(d[8] | d[16] | d[24] | d[32] | d[40] | d[48] | d[56])) {
                for (int r = 0; r < 8; r++) tmp[r * 8 + c] = d[0] * 4;
                continue;
            }
            int ev[4], od[4];
            even_odd(d[0], d[8], d[16], d[24], d[32], d[40], d[48], d[56], ev, od);
            for (int i = 0; i < 4; i++) {
                tmp[i * 8 + c] = (ev[i] + 512 + od[i]) >> 10;
                tmp[(7 - i) * 8 + c] = (ev[i] + 512 - od[i]) >> 10;
            }
        }
        for (int r = 0; r < 8; r++) {
            const int *v = tmp + r * 8;
            int ev[4], od[4];
            even_odd(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], ev, od);
            uint8_t *o = out + static_cast<size_t>(r) * stride;
            const int bias = 65536 + (128 << 17);
            for (int i = 0; i < 4; i++) {
                o[i] = clamp255((ev[i] + bias + od[i]) >> 17);
                o[7 - i] = clamp255((ev[i] + bias - od[i]) >> 17);
            }
        }
    }

    bool run(const uint8_t *data, size_t size) {
        p = data;
        end = data + size;
        if (u8() != 0xff || u8() != 0xd8) return fail("not a JPEG file");
        bool frame = false;
        while (p < end) {
            if (u8() != 0xff) return fail("bad JPEG marker");
            int m = u8();
            while (m == 0xff) m = u8();
            if (m == 0xd9) break;  // EOI
            if (m >= 0xd0 && m <= 0xd7) continue;
            const int len = u16() - 2;
            if (len < 0 || p + len > end) return fail("truncated JPEG segment");
            const uint8_t *next = p + len;
            if (m == 0xc4) {
                if (!read_dht(len)) return false;
            } else if (m == 0xdb) {
                if (!read_dqt(len)) return false;
            } else if (m == 0xc0 || m == 0xc1) {
                if (!read_sof(len)) return false;
                frame = true;
            } else if ((m >= 0xc2 && m <= 0xcf) && m != 0xc4 && m != 0xc8 && m != 0xcc) {
                return fail(m == 0xc2 ? "progressive JPEG is not read" : "unsupported JPEG coding");
            } else if (m == 0xdd) {
                restart = u16();
            } else if (m == 0xda) {
                if (!frame) return fail("JPEG scan before the frame header");
                if (!read_sos()) return false;
                continue;  // p is at the next marker
            } else if (m == 0xe0) {
                jfif = len >= 5 && !std::memcmp(p, "JFIF\0", 5);
            } else if (m == 0xee) {
                if (len >= 12 && !std::memcmp(p, "Adobe", 5)) adobe_transform = p[11];
            }
            p = next;
        }
        return frame || fail("JPEG without a frame");
    }
};

// One output row of component c upsampled to the image width (the filter stb chooses for its factors).
void upsample_row(int hs, int vs, const uint8_t *near_row, const uint8_t *far_row, int w_lores, uint8_t *out) {
    auto div4 = [](int x) { return static_cast<uint8_t>(x >> 2); };
    auto div16 = [](int x) { return static_cast<uint8_t>(x >> 4); };
    if (hs == 1 && vs == 1) {
        std::memcpy(out, near_row, w_lores);
    } else if (hs == 1 && vs == 2) {
        for (int i = 0; i < w_lores; i++) out[i] = div4(3 * near_row[i] + far_row[i] + 2);
    } else if (hs == 2 && vs == 1) {
        const uint8_t *in = near_row;
        if (w_lores == 1) {
            out[0] = out[1] = in[0];
            return;
        }
        out[0] = in[0];
        out[1] = div4(in[0] * 3 + in[1] + 2);
        int i = 1;
        for (; i < w_lores - 1; i++) {
            const int n = 3 * in[i] + 2;
            out[2 * i] = div4(n + in[i - 1]);
            out[2 * i + 1] = div4(n + in[i + 1]);
        }
        out[2 * i] = div4(in[w_lores - 2] * 3 + in[w_lores - 1] + 2);
        out[2 * i + 1] = in[w_lores - 1];
    } else if (hs == 2 && vs == 2) {
        if (w_lores == 1) {
            out[0] = out[1] = div4(3 * near_row[0] + far_row[0] + 2);
            return;
        }
        int t1 = 3 * near_row[0] + far_row[0];
        out[0] = div4(t1 + 2);
        for (int i = 1; i < w_lores; i++) {
            const int t0 = t1;
            t1 = 3 * near_row[i] + far_row[i];
            out[2 * i - 1] = div16(3 * t0 + t1 + 8);
            out[2 * i] = div16(3 * t1 + t0 + 8);
        }
        out[2 * w_lores - 1] = div4(t1 + 2);
    } else {
        for (int i = 0; i < w_lores; i++)
            for (int j = 0; j < hs; j++) out[i * hs + j] = near_row[i];
    }
}

}  // namespace

// Decodes a baseline JPEG into 8-bit samples: comps 1 (gray) or 3 (RGB).  False with err on failure.
bool decode_jpeg(const std::vector<uint8_t> &f, int comps, std::vector<uint8_t> &px, int &W, int &H,
                 std::string &err) {
    Decoder dec;
    if (!dec.run(f.data(), f.size())) {
        err = dec.err;
        return false;
    }
    W = dec.W;
    H = dec.H;
    const int n_in = static_cast<int>(dec.comp.size());
    const bool is_rgb = n_in == 3 && ((dec.comp[0].id == 'R' && dec.comp[1].id == 'G' && dec.comp[2].id == 'B') ||
                                      (dec.adobe_transform == 0 && !dec.jfif));
    // components needed: the Y plane alone for gray output of a YCbCr image
    const int decode_n = (n_in == 3 && comps < 3 && !is_rgb) ? 1 : n_in;
    struct Res {
        int hs, vs, ystep, w_lores, ypos, rows;
        const uint8_t *line0, *line1;
        int pitch;
        std::vector<uint8_t> buf;
    };
    std::vector<Res> res(decode_n);
    for (int k = 0; k < decode_n; k++) {
        const Component &c = dec.comp[k];
        Res &r = res[k];
        r.hs = dec.hmax / c.h;
        r.vs = dec.vmax / c.v;
        r.ystep = r.vs >> 1;
        r.w_lores = (W + r.hs - 1) / r.hs;
        r.ypos = 0;
        r.rows = (H * c.v + dec.vmax - 1) / dec.vmax;
        r.pitch = c.bw * 8;
        r.line0 = r.line1 = c.data.data();
        r.buf.assign(static_cast<size_t>(W) + 3 + 8, 0);
    }
    px.assign(static_cast<size_t>(W) * H * comps, 0);
    std::vector<const uint8_t *> row(decode_n);
    for (int y = 0; y < H; y++) {
        for (int k = 0; k < decode_n; k++) {
            Res &r = res[k];
            const bool bot = r.ystep >= (r.vs >> 1);
            upsample_row(r.hs, r.vs, bot ? r.line1 : r.line0, bot ? r.line0 : r.line1, r.w_lores, r.buf.data());
            row[k] = r.buf.data();
            if (++r.ystep >= r.vs) {
                r.ystep = 0;
                r.line0 = r.line1;
                if (++r.ypos < r.rows) r.line1 += r.pitch;
            }
        }
        uint8_t *out = &px[static_cast<size_t>(y) * W * comps];
        for (int x = 0; x < W; x++) {
            int rgb[3];
            if (decode_n == 1) {
                rgb[0] = rgb[1] = rgb[2] = row[0][x];
            } else if (is_rgb) {
                rgb[0] = row[0][x];
                rgb[1] = row[1][x];
                rgb[2] = row[2][x];
            } else {
                const int yf = (row[0][x] << 20) + (1 << 19);
                const int cr = row[2][x] - 128, cb = row[1][x] - 128;
                auto f2f = [](float v) { return static_cast<int>(v * 4096.0f + 0.5f) << 8; };
                rgb[0] = (yf + cr * f2f(1.40200f)) >> 20;
                rgb[1] = (yf + cr * -f2f(0.71414f) + static_cast<int>(static_cast<unsigned>(cb * -f2f(0.34414f)) &
                                                                      0xffff0000u)) >> 20;
                rgb[2] = (yf + cb * f2f(1.77200f)) >> 20;
                for (int& v : rgb) v = v < 0 ? 0 : (v > 255 ? 255 : v);
            }
            if (comps == 1)
                out[x] = (decode_n == 1) ? static_cast<uint8_t>(rgb[0])
                                         : static_cast<uint8_t>(((rgb[0] * 77) + (rgb[1] * 150) + (29 * rgb[2])) >> 8);
            else
                for (int k = 0; k < 3; k++) out[3 * x + k] = static_cast<uint8_t>(rgb[k]);
        }
    }
    return true;
}

}  // namespace lpaici_cli
