// tile_core.cuh -- the per-tile LPA-ICI forward sweep shared by the single-image and the batched
// (persistent) kernels.
//
// Layout of one CTA's shared memory:
//   blob   the packed kernel set (BlobLayout): run ranges, Run records, weights
//   tab    var[nk], thr[nk] of the image being processed
//   tile   (TH + 2R) rows x pitch floats: the input window of the output tile plus a halo of R rows
//          above/below, HL = align4(R) columns left and >= R right; zero outside the image
//
// Thread mapping: a warp covers 8 rows x (4 lanes x P) columns; lane = 4*row + quarter.  Each
// thread owns P horizontally adjacent pixels.  With P odd and pitch/4 odd the 32 lanes of a scalar
// shared-memory load hit 32 different banks (rows give the 8 multiples of 4, the lane's column
// offset quarter*P gives the 4 residues mod 4).
//
// Arithmetic (bit-identical to src/v1_0_lpa_ici_2D_fused.cpp:803-930 for finite inputs):
//   conv  = sum over the kernel's taps in row-major order of __fmul_rn(w, x), added with __fadd_rn,
//           starting from +0.0f; zero-filled halo taps add +-0, which changes nothing (a running sum
//           started at +0 never becomes -0);
//   lb/ub = conv -+ thr;  lo = max(lo, lb); hi = min(hi, ub); accept while hi >= lo, else stop;
//   num  += est * (1/var); den += 1/var (in direction order);  out = num / den.
#pragma once

#include "internal.h"

namespace lpaici {

// Smallest pitch >= need with pitch % 4 == 0 and (pitch / 4) odd (conflict-free rows, 16 B rows).
__host__ __device__ inline int tile_pitch(int need) {
    int p = (need + 3) & ~3;
    if (((p >> 2) & 1) == 0) p += 4;
    return p;
}

template <int P, int WX, int WY>
struct TileShape {
    static constexpr int kPixels = P;
    static constexpr int kThreads = 32 * WX * WY;
    static constexpr int kTileW = WX * 4 * P;
    static constexpr int kTileH = WY * 8;
};

// Smem geometry of a tile for radius R.
struct TileGeom {
    int HL, pitch, rows;
    __host__ __device__ static TileGeom make(int tile_w, int tile_h, int R) {
        TileGeom g;
        g.HL = (R + 3) & ~3;
        g.pitch = tile_pitch(g.HL + tile_w + R);
        g.rows = tile_h + 2 * R;
        return g;
    }
};

// acc[i] += sum_{j < len} w[j] * src[i + j], for the P pixels of a thread, tap by tap in order.
// The window holds src[m] in slot m % P; every step loads one new value.
template <int P>
__device__ __forceinline__ void conv_run(float (&acc)[P], const float *__restrict__ src, const float *__restrict__ w,
                                         int len) {
    float win[P];
#pragma unroll
    for (int i = 0; i < P - 1; i++) win[i] = src[i];
    int k = 0;
    for (; k + P <= len; k += P) {
#pragma unroll
        for (int j = 0; j < P; j++) {
            win[(j + P - 1) % P] = src[k + j + P - 1];
            const float wt = w[k + j];
#pragma unroll
            for (int i = 0; i < P; i++) acc[i] = __fadd_rn(acc[i], __fmul_rn(wt, win[(j + i) % P]));
        }
    }
#pragma unroll
    for (int j = 0; j < P - 1; j++) {
        if (k + j < len) {
            win[(j + P - 1) % P] = src[k + j + P - 1];
            const float wt = w[k + j];
#pragma unroll
            for (int i = 0; i < P; i++) acc[i] = __fadd_rn(acc[i], __fmul_rn(wt, win[(j + i) % P]));
        }
    }
}

// Copies `words` 32-bit words (a multiple of 4, 16-byte aligned) from global to shared memory.
__device__ __forceinline__ void stage_words(int *dst, const int *__restrict__ src, int words) {
    const int4 *s = reinterpret_cast<const int4 *>(src);
    int4 *d = reinterpret_cast<int4 *>(dst);
    for (int i = threadIdx.x; i < (words >> 2); i += blockDim.x) d[i] = __ldg(s + i);
}

// Loads the halo'd input window of the output tile whose top-left output pixel is (x0, y0).
// Input pixel (gy, gx) with gy = y0 + row_begin - R + r, gx = x0 - HL + c; zero outside the input.
__device__ __forceinline__ void load_tile(float *s_tile, const ImageArgs &img, int x0, int y0, int R,
                                          const TileGeom &g) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int gy0 = y0 + img.row_begin - R, gx0 = x0 - g.HL;
    for (int r = warp; r < g.rows; r += nwarps) {
        const int gy = gy0 + r;
        const bool row_ok = gy >= 0 && gy < img.in_h;
        const float *src = img.in + static_cast<size_t>(row_ok ? gy : 0) * img.in_pitch;
        float *dst = s_tile + r * g.pitch;
        for (int c = lane; c < g.pitch; c += 32) {
            const int gx = gx0 + c;
            dst[c] = (row_ok && gx >= 0 && gx < img.W) ? __ldg(src + gx) : 0.0f;
        }
    }
}

// Lane geometry of a thread inside its tile.
template <int P, int WX>
struct LaneGeom {
    int ty, tx;  // tile-local row and first column of the thread's P pixels
    __device__ __forceinline__ LaneGeom() {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        ty = (warp / WX) * 8 + (lane >> 2);
        tx = (warp % WX) * 4 * P + (lane & 3) * P;
    }
};

// The ICI scale sweep of one direction d for the thread's P pixels (mask `valid`): for every
// pixel the estimate, variance and index of the last accepted scale.  Warp-uniform loop over the
// scales; it ends when every pixel of the warp has stopped.
template <int P>
__device__ __forceinline__ void direction_sweep(int d, int S, unsigned valid, const float *lane_tile, int pitch,
                                                const int *s_blob, const int4 *s_runs, const float *s_w,
                                                const float *s_var, const float *s_thr, float (&best)[P],
                                                float (&bvar)[P], int (&sidx)[P]) {
    float lo[P], hi[P];
#pragma unroll
    for (int i = 0; i < P; i++) {
        lo[i] = -INFINITY;
        hi[i] = INFINITY;
        best[i] = 0.0f;
        bvar[i] = 0.0f;
        sidx[i] = 0;
    }
    unsigned alive = valid;
    for (int s = 0; s < S; s++) {
        if (!__any_sync(0xffffffffu, alive)) break;  // every pixel of the warp has stopped
        const int k = d * S + s;
        float acc[P];
#pragma unroll
        for (int i = 0; i < P; i++) acc[i] = 0.0f;
        const int rb = s_blob[k], re = s_blob[k + 1];
        for (int r = rb; r < re; r++) {
            const int4 run = s_runs[r];
            conv_run<P>(acc, lane_tile + run.x * pitch + run.y, s_w + run.w, run.z);
        }
        const float thr = s_thr[k], var = s_var[k];
#pragma unroll
        for (int i = 0; i < P; i++) {
            if (alive & (1u << i)) {
                const float lb = __fsub_rn(acc[i], thr);
                const float ub = __fadd_rn(acc[i], thr);
                lo[i] = fmaxf(lo[i], lb);
                hi[i] = fminf(hi[i], ub);
                if (hi[i] >= lo[i]) {
                    best[i] = acc[i];
                    bvar[i] = var;
                    sidx[i] = s;
                } else {
                    alive &= ~(1u << i);
                }
            }
        }
    }
}

// The forward sweep of one tile (tile already in shared memory, block-synchronised).
template <int P, int WX, int WY>
__device__ __forceinline__ void sweep_tile(const ImageArgs &img, int x0, int y0, int D, int S, int R,
                                           const TileGeom &g, const int *s_blob, int run_word, int weight_word,
                                           const float *s_var, const float *s_thr, const float *s_tile) {
    const LaneGeom<P, WX> lg;
    const int oy = y0 + lg.ty, ox = x0 + lg.tx;
    unsigned valid = 0;
    if (oy < img.rows_out) {
#pragma unroll
        for (int i = 0; i < P; i++)
            if (ox + i < img.W) valid |= 1u << i;
    }
    const float *lane_tile = s_tile + (lg.ty + R) * g.pitch + lg.tx + g.HL;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + run_word);
    const float *s_w = reinterpret_cast<const float *>(s_blob + weight_word);

    float num[P], den[P];
#pragma unroll
    for (int i = 0; i < P; i++) num[i] = den[i] = 0.0f;

    for (int d = 0; d < D; d++) {
        float best[P], bvar[P];
        int sidx[P];
        direction_sweep<P>(d, S, valid, lane_tile, g.pitch, s_blob, s_runs, s_w, s_var, s_thr, best, bvar, sidx);
#pragma unroll
        for (int i = 0; i < P; i++) {
            const float rcp = __fdiv_rn(1.0f, bvar[i]);
            num[i] = __fadd_rn(num[i], __fmul_rn(best[i], rcp));
            den[i] = __fadd_rn(den[i], rcp);
        }
        if (img.smap) {
            uint8_t *m = img.smap + (static_cast<size_t>(d) * img.rows_out + oy) * img.W + ox;
#pragma unroll
            for (int i = 0; i < P; i++)
                if (valid & (1u << i)) m[i] = static_cast<uint8_t>(sidx[i]);
        }
    }
    float *o = img.out + static_cast<size_t>(oy) * img.out_pitch + ox;
#pragma unroll
    for (int i = 0; i < P; i++)
        if (valid & (1u << i)) o[i] = __fdiv_rn(num[i], den[i]);
}

}  // namespace lpaici
