// tile_core.cuh -- the per-tile LPA-ICI sweep shared by the single-image, batched and adjoint kernels.
//
// Shared memory of one CTA:
//   blob   the packed kernel set (BlobLayout): run ranges, Run records, duplicated weights {w, w}
//   tab    var[nk], thr[nk], rvar[nk] = 1/var of the image being processed
//   tile   T8[j][c] = {x(j, c), x(j + 8, c)}: the input window of the output tile as pairs of rows
//          8 apart, j < TH - 8 + 2R, c < pitch2 (odd); input row j is output row j - R of the tile,
//          input column c is output column c - R; zero outside the input
//
// Thread mapping (Q = column pairs per thread, 4 or 8): a warp covers 16 rows x 4Q columns; the lane
// with row index a (0..7) and column group b (0..3) owns the 2Q pixels of rows (a, a + 8) and columns
// Qb .. Qb + Q - 1, held as Q float2 pairs {row a, row a + 8}.  Every window value is then a natural
// register pair, so one packed product and one packed add do two pixels' taps.  The 16 lanes of a
// half-warp hit 16 different bank pairs with 8-byte loads (pitch2 odd): Q = 4 puts 4 rows x 4 groups
// in a half-warp (rows give the residues mod 4, groups the multiples of 4), Q = 8 puts 8 rows x 2
// groups (rows give 8 distinct values mod 16 that never differ by 8, groups add 0 or 8).
//
// Arithmetic (bit-identical to src/v1_0_lpa_ici_2D_fused.cpp:803-930 for finite inputs):
//   conv  = sum over the kernel's taps in row-major order of w*x (rounded), added one by one with
//           round-to-nearest, starting from +0.0f -- packed f32x2 instructions round each half on its
//           own; zero-filled halo taps and zero weights add +-0, which changes nothing (a running sum
//           started at +0 never becomes -0);
//   lb/ub = conv -+ thr;  lo = max(lo, lb); hi = min(hi, ub); accept while hi >= lo, else stop;
//   num  += est * (1/var); den += 1/var (in direction order, 1/var correctly rounded);  out = num / den.
#pragma once

#include <type_traits>

#include "internal.h"

namespace lpaici {

// Packed FP32 arithmetic, two lanes per instruction, each half rounded to nearest on its own.
//
// ptxas contracts a packed multiply feeding a packed add (mul.rn.f32x2 -> add.rn.f32x2) into one
// fused multiply-add even with .rn and --fmad=false, which changes the rounding of the sums.  The
// product is therefore formed as fma.rn.f32x2(w, x, nz) with nz = {-0, -0} passed in at run time
// (so it cannot be folded away): w*x + (-0) is w*x exactly before the single rounding, hence the
// correctly rounded product with its sign of zero; an fma feeding an add is never contracted.
__device__ __forceinline__ float2 prod2(float2 a, float2 b, float2 nz) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(nz.x), "f"(nz.y));
    return d;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// One tap of the forward: the product rounded, then the sum rounded (bit-exact with the reference).
struct ExactTap {
    float2 nz;  // {-0, -0}, read at run time (see prod2)
    __device__ __forceinline__ float2 operator()(float2 acc, float2 w, float2 x) const {
        return add2(acc, prod2(w, x, nz));
    }
};

// d = a * b + c in each half, rounded on its own (the two halves of fmaf).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// One tap as a fused multiply-add, acc + w * x rounded once: the adjoint's gather, and the forward's
// contracted mode (not bit-exact with the reference).
struct FmaTap {
    __device__ __forceinline__ float2 operator()(float2 acc, float2 w, float2 x) const { return fma2(w, x, acc); }
};

// Smallest odd pitch (in float2) >= need.
__host__ __device__ inline int tile_pitch2(int need) { return need | 1; }

template <int WX, int WY, int Q>
struct TileShape {
    static constexpr int kThreads = 32 * WX * WY;
    static constexpr int kTileW = WX * 4 * Q;
    static constexpr int kTileH = WY * 16;
};

// Shared-memory geometry of a tile for radius R and Q column pairs per thread: tile_w + 2R columns
// of halo'd input plus Q spare columns, a margin no load reaches (the last column a run's window
// reads is tile_w + 2R - 1).
struct TileGeom {
    int R, pitch2, pairs;  // pairs: number of T8 rows
    __host__ __device__ static TileGeom make(int tile_w, int tile_h, int R, int Q) {
        TileGeom g;
        g.R = R;
        g.pitch2 = tile_pitch2(tile_w + 2 * R + Q);
        g.pairs = tile_h - 8 + 2 * R;
        return g;
    }
    __host__ __device__ size_t tile_bytes() const { return sizeof(float2) * static_cast<size_t>(pitch2) * pairs; }
};

// Words of shared memory before the tile: the blob, then var/thr/rvar (padded to 16 bytes).
__host__ __device__ inline int table_words(int nk) { return (3 * nk + 3) & ~3; }

// One tap column J of a block of Q: window slot (J + Q - 1) % Q receives column k + J + Q - 1, then
// the Q pixel pairs m accumulate w * column (k + J + m) with the tap operation.  Weights come two taps
// per float4.
#define LPAICI_STEP(J)                                                                               \
    {                                                                                                \
        if (((J) & 1) == 0) wv = wq[(J) >> 1];                                                       \
        const float2 w2 = ((J) & 1) ? make_float2(wv.z, wv.w) : make_float2(wv.x, wv.y);             \
        win[((J) + Q - 1) % Q] = src[(J) + Q - 1];                                                   \
        _Pragma("unroll") for (int m = 0; m < Q; m++) acc[m] = tap(acc[m], w2, win[((J) + m) % Q]);  \
    }

// The last N (< Q) taps of a run: their window columns and weights are loaded before any of them is
// used, so the tail pays no load latency per tap.  Win: a pointer to the run's first column pair, or a
// window type with the same indexing (the adjoint's masked field).
template <int Q, int N, class Win, class Tap>
__device__ __forceinline__ void conv_tail(float2 (&acc)[Q], float2 (&win)[Q], const Win &src,
                                          const float4 *__restrict__ wq, const Tap &tap) {
    float2 tail[N];
    float4 tw[(N + 1) / 2];
#pragma unroll
    for (int J = 0; J < N; J++) tail[J] = src[J + Q - 1];
#pragma unroll
    for (int i = 0; i < (N + 1) / 2; i++) tw[i] = wq[i];
#pragma unroll
    for (int J = 0; J < N; J++) {
        const float2 w2 = (J & 1) ? make_float2(tw[J >> 1].z, tw[J >> 1].w) : make_float2(tw[J >> 1].x, tw[J >> 1].y);
        win[(J + Q - 1) % Q] = tail[J];
#pragma unroll
        for (int m = 0; m < Q; m++) acc[m] = tap(acc[m], w2, win[(J + m) % Q]);
    }
}

template <int Q, class Win, class Tap>
__device__ __forceinline__ void conv_tail_dispatch(int rem, float2 (&acc)[Q], float2 (&win)[Q], const Win &src,
                                                   const float4 *__restrict__ wq, const Tap &tap) {
    if constexpr (Q == 4) {
        switch (rem) {
            case 1: conv_tail<Q, 1>(acc, win, src, wq, tap); break;
            case 2: conv_tail<Q, 2>(acc, win, src, wq, tap); break;
            default: conv_tail<Q, 3>(acc, win, src, wq, tap); break;
        }
    } else {
        static_assert(Q == 8, "tile configurations use Q = 4 or 8");
        switch (rem) {
            case 1: conv_tail<Q, 1>(acc, win, src, wq, tap); break;
            case 2: conv_tail<Q, 2>(acc, win, src, wq, tap); break;
            case 3: conv_tail<Q, 3>(acc, win, src, wq, tap); break;
            case 4: conv_tail<Q, 4>(acc, win, src, wq, tap); break;
            case 5: conv_tail<Q, 5>(acc, win, src, wq, tap); break;
            case 6: conv_tail<Q, 6>(acc, win, src, wq, tap); break;
            default: conv_tail<Q, 7>(acc, win, src, wq, tap); break;
        }
    }
}

// acc[m] = tap(acc[m], {w_j, w_j}, src[m + j]) for j < len, tap by tap in order, for the Q pixel pairs.
// src: the run's first column in T8 (row already chosen); wq: the run's duplicated weights as
// float4 {w_2i, w_2i, w_2i+1, w_2i+1}.
// The last len % Q taps go to a tail of exactly that many taps (conv_tail): one warp-uniform
// dispatch, no test per tap.  src and wq advance with the taps, so every load has a constant offset.
template <int Q, class Win, class Tap>
__device__ __forceinline__ void conv_run(float2 (&acc)[Q], Win src, const float4 *__restrict__ wq, int len,
                                         const Tap &tap) {
    float2 win[Q];
    float4 wv;
#pragma unroll
    for (int i = 0; i < Q - 1; i++) win[i] = src[i];
    int rem = len;
    for (; rem >= Q; rem -= Q, src += Q, wq += Q / 2) {
#pragma unroll
        for (int J = 0; J < Q; J++) LPAICI_STEP(J)
    }
    // rem: 0 .. Q-1, warp-uniform: one dispatch to a tail of exactly rem taps
    if (rem > 0) conv_tail_dispatch<Q>(rem, acc, win, src, wq, tap);
}
#undef LPAICI_STEP

// Copies `words` 32-bit words (a multiple of 4, 16-byte aligned) from global to shared memory.
__device__ __forceinline__ void stage_words(int *dst, const int *__restrict__ src, int words) {
    const int4 *s = reinterpret_cast<const int4 *>(src);
    int4 *d = reinterpret_cast<int4 *>(dst);
    for (int i = threadIdx.x; i < (words >> 2); i += blockDim.x) d[i] = __ldg(s + i);
}

// Copies the forward blob like stage_words and rewrites each run (row, col, len, w) on the way into
// (row * pitch2 + col, len, w / 2, 0): its first input pair as an offset into the tile and its first
// duplicated weight pair as a float4 index.  Runs occupy words [run_word, weight_word).
__device__ __forceinline__ void stage_blob(int *dst, const int *__restrict__ src, int words, int run_word,
                                           int weight_word, int pitch2) {
    const int4 *s = reinterpret_cast<const int4 *>(src);
    int4 *d = reinterpret_cast<int4 *>(dst);
    const int r0 = run_word >> 2, r1 = weight_word >> 2;
    for (int i = threadIdx.x; i < (words >> 2); i += blockDim.x) {
        int4 v = __ldg(s + i);
        if (i >= r0 && i < r1) v = make_int4(v.x * pitch2 + v.y, v.z, v.w >> 1, 0);
        d[i] = v;
    }
}

// var, thr and rvar = 1/var (correctly rounded, the reference's 1.0f / var_d) into shared memory.
__device__ __forceinline__ void stage_tables(float *s_tab, const float *var, const float *thr, int nk) {
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
        s_tab[i] = var[i];
        s_tab[nk + i] = thr[i];
        s_tab[2 * nk + i] = __fdiv_rn(1.0f, var[i]);
    }
}

// Builds T8 for the output tile whose top-left output pixel is (x0, y0): input pixel
// (gy0 + j, gx0 + c) and (gy0 + j + 8, gx0 + c), gy0 = y0 + row_begin - R, gx0 = x0 - R.
__device__ __forceinline__ void load_tile(float2 *s_tile, const ImageArgs &img, int x0, int y0, const TileGeom &g) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int gy0 = y0 + img.row_begin - g.R, gx0 = x0 - g.R;
    for (int j = warp; j < g.pairs; j += nwarps) {
        const int ga = gy0 + j, gb = ga + 8;
        const bool ok_a = ga >= 0 && ga < img.in_h, ok_b = gb >= 0 && gb < img.in_h;
        const float *ra = img.in + static_cast<size_t>(ok_a ? ga : 0) * img.in_pitch;
        const float *rb = img.in + static_cast<size_t>(ok_b ? gb : 0) * img.in_pitch;
        float2 *dst = s_tile + j * g.pitch2;
        for (int c = lane; c < g.pitch2; c += 32) {
            const int gx = gx0 + c;
            const bool ok_x = gx >= 0 && gx < img.W;
            const size_t at = static_cast<size_t>(gx) * img.step;
            dst[c] = make_float2(ok_a && ok_x ? __ldg(ra + at) : 0.0f, ok_b && ok_x ? __ldg(rb + at) : 0.0f);
        }
    }
}

// Lane geometry inside the tile: rows ty and ty + 8, columns tx .. tx + Q - 1 (tile-local output).
template <int WX, int Q>
struct LaneGeom {
    int ty, tx;
    __device__ __forceinline__ LaneGeom() {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int a = Q == 4 ? (lane >> 2) : (lane & 7), b = Q == 4 ? (lane & 3) : (lane >> 3);
        ty = (warp / WX) * 16 + a;
        tx = (warp % WX) * 4 * Q + Q * b;
    }
};

// Pixel i = 2m + h of a thread: column tx + m, row ty + 8h.
template <int Q>
__device__ __forceinline__ float pick(const float2 (&v)[Q], int i) { return (i & 1) ? v[i >> 1].y : v[i >> 1].x; }

// Per-thread selected-scale indices, 4 bits per pixel.
template <int Q>
using ScaleBits = typename std::conditional<(8 * Q <= 32), unsigned, unsigned long long>::type;

// The ICI scale sweep of direction d for the thread's 2Q pixels (mask `valid`): per pixel the estimate
// of the last accepted scale (best) and that scale's index (sidx, 4 bits per pixel).  The intersection
// [lo, hi] only shrinks, so once it is empty no later scale can be accepted: a stopped pixel needs no
// mask, its updates simply never accept again.  Scale 0 is always accepted (lo = -inf, hi = +inf), so
// the index is the count of accepted scales after it.  Warp-uniform scale loop; it ends when every
// valid pixel of the warp has stopped.
template <int Q, bool Fused>
__device__ __forceinline__ void direction_sweep(int d, int S, unsigned valid, const float2 *lane_tile,
                                                const int *s_blob, const int4 *s_runs, const float4 *s_wq,
                                                const float *s_thr, float2 nz, float2 (&best)[Q], ScaleBits<Q> &sidx) {
    float lo[2 * Q], hi[2 * Q];
#pragma unroll
    for (int i = 0; i < 2 * Q; i++) {
        lo[i] = -INFINITY;
        hi[i] = INFINITY;
    }
#pragma unroll
    for (int m = 0; m < Q; m++) best[m] = make_float2(0.0f, 0.0f);
    sidx = 0;
    bool alive = valid != 0;
    for (int s = 0; s < S; s++) {
        if (!__any_sync(0xffffffffu, alive)) break;  // every valid pixel of the warp has stopped
        const int k = d * S + s;
        float2 acc[Q];
#pragma unroll
        for (int m = 0; m < Q; m++) acc[m] = make_float2(0.0f, 0.0f);
        const int rb = s_blob[k], re = s_blob[k + 1];
        // two runs per iteration for Q = 4: the compiler then keeps the 768-thread tiles within 80
        // registers without spilling (measured: 24 warps per SM beat 20)
#pragma unroll(Q == 4 ? 2 : 1)
        for (int r = rb; r < re; r++) {
            const int4 run = s_runs[r];  // (tile offset, len, float4 weight index): see stage_blob
            if constexpr (Fused)
                conv_run<Q>(acc, lane_tile + run.x, s_wq + run.z, run.y, FmaTap{});
            else
                conv_run<Q>(acc, lane_tile + run.x, s_wq + run.z, run.y, ExactTap{nz});
        }
        const float thr = s_thr[k];
        const ScaleBits<Q> step = s > 0 ? 1 : 0;
        float2 lb[Q], ub[Q];
#pragma unroll
        for (int m = 0; m < Q; m++) {
            lb[m] = add2(acc[m], make_float2(-thr, -thr));  // conv - thr, exactly
            ub[m] = add2(acc[m], make_float2(thr, thr));
        }
        alive = false;
#pragma unroll
        for (int i = 0; i < 2 * Q; i++) {
            lo[i] = fmaxf(lo[i], pick<Q>(lb, i));
            hi[i] = fminf(hi[i], pick<Q>(ub, i));
            const bool ok = hi[i] >= lo[i];
            if (i & 1)
                best[i >> 1].y = ok ? acc[i >> 1].y : best[i >> 1].y;
            else
                best[i >> 1].x = ok ? acc[i >> 1].x : best[i >> 1].x;
            sidx += ok ? static_cast<ScaleBits<Q>>(step << (4 * i)) : ScaleBits<Q>(0);
            alive |= ok && ((valid >> i) & 1u);
        }
    }
}

// The forward sweep of one tile (tile in shared memory, block-synchronised).
template <int WX, int Q, bool Fused = false>
__device__ __forceinline__ void sweep_tile(const ImageArgs &img, int x0, int y0, int D, int S, const TileGeom &g,
                                           const int *s_blob, int run_word, int weight_word, const float *s_tab,
                                           const float2 *s_tile, float neg_zero) {
    const LaneGeom<WX, Q> lg;
    const int nk = D * S;
    const int oy = y0 + lg.ty, ox = x0 + lg.tx;
    unsigned valid = 0;
#pragma unroll
    for (int i = 0; i < 2 * Q; i++)
        if (oy + 8 * (i & 1) < img.rows_out && ox + (i >> 1) < img.W) valid |= 1u << i;
    const float2 *lane_tile = s_tile + (lg.ty + g.R) * g.pitch2 + lg.tx + g.R;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + run_word);
    const float4 *s_wq = reinterpret_cast<const float4 *>(s_blob + weight_word);
    const float *s_thr = s_tab + nk, *s_rvar = s_tab + 2 * nk;
    const float2 nz = make_float2(neg_zero, neg_zero);

    float2 num[Q], den[Q];
#pragma unroll
    for (int m = 0; m < Q; m++) num[m] = den[m] = make_float2(0.0f, 0.0f);

    for (int d = 0; d < D; d++) {
        float2 best[Q];
        ScaleBits<Q> sidx;
        direction_sweep<Q, Fused>(d, S, valid, lane_tile, s_blob, s_runs, s_wq, s_thr, nz, best, sidx);
#pragma unroll
        for (int m = 0; m < Q; m++) {
            const float2 r = make_float2(s_rvar[d * S + static_cast<int>((sidx >> (8 * m)) & 15)],
                                         s_rvar[d * S + static_cast<int>((sidx >> (8 * m + 4)) & 15)]);
            num[m] = add2(num[m], prod2(best[m], r, nz));
            den[m] = add2(den[m], r);
        }
        if (img.smap) {
#pragma unroll
            for (int i = 0; i < 2 * Q; i++)
                if (valid & (1u << i))
                    img.smap[(static_cast<size_t>(d) * img.rows_out + oy + 8 * (i & 1)) * img.W + ox + (i >> 1)] =
                        static_cast<uint8_t>((sidx >> (4 * i)) & 15);
        }
    }
    if (img.out) {
#pragma unroll
        for (int i = 0; i < 2 * Q; i++)
            if (valid & (1u << i))
                img.out[static_cast<size_t>(oy + 8 * (i & 1)) * img.out_pitch +
                        static_cast<size_t>(ox + (i >> 1)) * img.step] =
                    __fdiv_rn(pick<Q>(num, i), pick<Q>(den, i));
    }
    if (img.rden) {
#pragma unroll
        for (int i = 0; i < 2 * Q; i++)
            if (valid & (1u << i))
                img.rden[static_cast<size_t>(oy + 8 * (i & 1)) * img.W + ox + (i >> 1)] = __frcp_rn(pick<Q>(den, i));
    }
}

}  // namespace lpaici
