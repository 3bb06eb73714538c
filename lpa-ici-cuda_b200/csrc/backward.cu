// backward.cu -- adjoint of the LPA-ICI forward with the ICI selection held fixed.
//
// For L = sum_p g[p] * out[p] and the selected scale s*(d,p) of every direction and pixel frozen,
// out is linear in the input x:  out(p) = sum_d alpha_d(p) * sum_t h_{d,s*}(t) x(p + t - c), with
// alpha_d(p) = (1/v_{d,s*}) / den(p), den(p) = sum_d' 1/v_{d',s*}.  With the adjoint field of direction d
//     c_d(p) = g(p) / den(p) / v_{d, s*(d,p)},
//     dL/dx(q) = sum_d sum_s sum_t h'_{d,s}(t) [s*(d, q + t) = s] c_d(q + t)       (zero padding)
// where h' is h mirrored through its centre: for every direction and scale, a correlation of the field
// masked to the pixels that selected that scale.  Three launches:
//   A. selection: the forward's exact tile sweep recomputes s*(d,p) (one byte per direction and
//      pixel) and 1/den(p) into a transient workspace -- the forward stores nothing for the adjoint;
//   u: u = g / den over the workspace's 1/den (an elementwise pass; from a kept state the gather forms
//      the product itself);
//   B. gather: one CTA per 128 x 64 output tile.  Per direction it reads s*(d,.) and u on the tile plus
//      its R-pixel halo (from L2) and forms the field c_d = u / v_{d,s*} in shared memory.
//      The kernels are telescoped, D_s = h'_s - h'_{s-1} (D_0 = h'_0, built by kernelset.cpp), which
//      turns the sum over scales into
//          sum_s D_s (*) (c_d [s* >= s]):
//      the field is zeroed in place where s* < s, scale after scale (only where the next kernel
//      reaches), and never rebuilt.  The runs are the forward's run loop (register sliding window over
//      Q columns, exact-length tails) with packed FMAs over two output rows -- the adjoint is checked
//      against FP64 finite differences, not bit patterns.  Groups of warps take every G-th run of each
//      kernel over the same outputs and add their sums in group order at the end.  Every output is
//      written once: no atomics, deterministic.
// No counterpart in the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

#include "configs.h"
#include "tile_core.cuh"

namespace lpaici {

namespace {

// Gather tile geometry.  A lane owns output rows ty and ty + 8 at Q = 8 consecutive columns and keeps
// them as the two halves of packed FMAs; a warp covers 16 rows x 32 columns: lane l has row index
// a = l & 7 and column group b = l >> 3.  The fields are plain row-major float arrays whose pitch p is
// 1 mod 8, so the 32 lanes' scalar loads of one row hit 32 different banks (a*p gives the residues
// mod 8, 8b the multiples of 8).  kGatherWX warps across and WY down make one group; G groups cover
// the same outputs, each with every G-th run of a kernel: four groups of up to 256 threads, else as
// many as make 1,024 threads.  Eight columns per lane spread each run's loop, window preload and tail
// over 16 outputs.
constexpr int kGatherQ = 8;
constexpr int kGatherPair = 8;  // rows between a lane's two output rows
constexpr int kGatherWX = 4;
constexpr int kGatherWarpCols = 32 / kGatherPair * kGatherQ;  // columns one warp covers
template <int WY>
struct GatherShape {
    static constexpr int kTW = kGatherWarpCols * kGatherWX;
    static constexpr int kTH = 2 * kGatherPair * WY;
    static constexpr int kGroupThreads = 32 * kGatherWX * WY;
    static constexpr int kG = kGroupThreads > 256 ? 1024 / kGroupThreads : 4;
    static constexpr int kThreads = kG * kGroupThreads;
};
// Tile heights the host can choose (the tallest whose field and kernels fit in shared memory): 128 x 64
// output tiles (two groups of 16 warps) for the 16 x 7 sets with radius 31.
constexpr int kGatherNWY = 4;
constexpr int kGatherWYs[kGatherNWY] = {4, 3, 2, 1};

// Field geometry: rows th + 2R, pitch 1 mod 8 and >= tw + 2R + Q (a margin no load reaches).
struct GatherGeom {
    int rows, pitch;
    __host__ __device__ static GatherGeom make(int tw, int th, int R) {
        GatherGeom g;
        g.rows = th + 2 * R;
        g.pitch = ((tw + 2 * R + kGatherQ + 6) & ~7) + 1;
        return g;
    }
    __host__ __device__ size_t cells() const { return static_cast<size_t>(rows) * pitch; }
    // cells rounded up to whole 4-cell words: the field and the scale map start 16-byte aligned, as the
    // masking's 16-byte accesses need
    __host__ __device__ size_t cells4() const { return (cells() + 3) & ~size_t(3); }
};

// Window of a run over a field: column i is the pair {a[i], b[i]} of the lane's two rows (b = a +
// kGatherPair rows).  Both pointers advance with the taps, so every load has a constant offset.
struct PairWin {
    const float *a, *b;
    __device__ __forceinline__ float2 operator[](int i) const { return make_float2(a[i], b[i]); }
    __device__ __forceinline__ PairWin &operator+=(int n) {
        a += n;
        b += n;
        return *this;
    }
};

// One image of the gather: pass A's outputs and the caller's buffers.
struct GatherImage {
    const float *g;        // cotangent, pitch g_pitch
    const uint8_t *smap;   // D x H x W selected scales (pass A)
    const float *rden;     // H x W, pitch W: 1 / den, den = sum_d 1/v_d (pass A); u = g / den when u_ready
    float *grad;           // result, pitch grad_pitch
    const float *rvar;     // 1 / v_k of this image (batched plans; one image: GatherArgs::rvar)
    int g_pitch, grad_pitch, W, H;
    int tiles_x;
    int u_ready;           // rden holds u = g * (1 / den) already (lpaici_adjoint_u_kernel)
};

struct GatherArgs {
    GatherImage single;          // the image of a one-image launch (images == null)
    const GatherImage *images;   // batched: per-image descriptors in device memory
    const int2 *items;           // batched: (image, tile) of every CTA
    int D, S, R;
    const int *blob;       // mirrored kernels (lpaici_kernelset::adj_blob, BlobLayout)
    int blob_words, run_word, weight_word;
    int pitch, rows;       // field geometry (GatherGeom of the tile)
    int th;                // output rows per tile
    float rvar[kMaxKernels];  // 1 / v_k of the one image
    // per kernel: the field cells its correlation reads, rows [x, y), columns [z, w); per direction: the
    // union over its scales (the cells its field needs)
    int4 rect[kMaxKernels];
    int4 drect[kMaxKernels];
};

// Shared memory: blob (runs as field offsets) | 1/v table | field | selected scales.
__host__ __device__ inline int rv_words(int nk) { return (nk + 3) & ~3; }
// The scale map carries 4 bytes past its last cell, set to 0xff: the masking reads it in whole words.
__host__ __device__ inline size_t gather_smem(int blob_words, int nk, const GatherGeom &g) {
    return sizeof(int) * (blob_words + rv_words(nk)) + sizeof(float) * g.cells4() + ((g.cells4() + 4 + 15) & ~size_t(15));
}

// Columns [c0, c1) of field row i0 / pitch of a direction's field build, lanes along the row: s*(d, .)
// into s_s and c_d = u / v_{d,s*} into s_f.  u is read from drow (UReady: u = g / den already) or formed
// as g * (1/den); cells outside the image get s* = 0 and u = 0.
template <bool UReady>
__device__ __forceinline__ void build_field_row(uint8_t *s_s, float *s_f, const float *rv_d, const uint8_t *prow,
                                                const float *grow, const float *drow, int i0, int c0, int c1, int gx0,
                                                int W, bool row_ok, int lane) {
    for (int c = c0 + lane; c < c1; c += 32) {
        const int gx = gx0 + c;
        unsigned sc = 0u;
        float u = 0.0f;
        if (row_ok && gx >= 0 && gx < W) {
            sc = __ldg(prow + gx);
            u = UReady ? __ldg(drow + gx) : __ldg(grow + gx) * __ldg(drow + gx);
        }
        s_s[i0 + c] = static_cast<uint8_t>(sc);
        s_f[i0 + c] = u * rv_d[sc];
    }
}

template <int WY>
__global__ void __launch_bounds__(GatherShape<WY>::kThreads, 1)
    lpaici_adjoint_gather_kernel(const __grid_constant__ GatherArgs a) {
    using Shape = GatherShape<WY>;
    constexpr int Q = kGatherQ, G = Shape::kG;
    extern __shared__ __align__(16) int smem[];
    const int nk = a.D * a.S;
    const int cells = a.rows * a.pitch, cells4 = (cells + 3) & ~3;
    int *s_blob = smem;
    float *s_rv = reinterpret_cast<float *>(smem + a.blob_words);
    float *s_f = s_rv + rv_words(nk);  // the field of the current direction
    uint8_t *s_s = reinterpret_cast<uint8_t *>(s_f + cells4);  // s*(d, .) on the halo'd tile
    GatherImage im;
    int tile = blockIdx.x;
    if (a.images) {
        const int2 it = a.items[blockIdx.x];
        im = a.images[it.x];
        tile = it.y;
    } else {
        im = a.single;
    }
    const float *rvar_k = a.images ? im.rvar : a.rvar;
    const int x0 = (tile % im.tiles_x) * Shape::kTW, y0 = (tile / im.tiles_x) * Shape::kTH;
    const int gx0 = x0 - a.R, gy0 = y0 - a.R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = Shape::kThreads >> 5;
    // the group is the same in every lane of a warp: reduced, the compiler knows it warp-uniform, so the
    // run loops and the tails' dispatch branch without reconvergence bookkeeping
    const int group = __reduce_max_sync(0xffffffffu, static_cast<unsigned>(threadIdx.x / Shape::kGroupThreads));
    const int gtid = threadIdx.x % Shape::kGroupThreads;
    const int gwarp = gtid >> 5;
    const int ty = (gwarp / kGatherWX) * 2 * kGatherPair + (lane & (kGatherPair - 1));  // and ty + kGatherPair
    const int tx = (gwarp % kGatherWX) * kGatherWarpCols + (lane / kGatherPair) * Q;
    const int lane_off = (ty + a.R) * a.pitch + tx + a.R;
    const int pair_rows = kGatherPair * a.pitch;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + a.run_word);
    const float4 *s_wq = reinterpret_cast<const float4 *>(s_blob + a.weight_word);

    stage_blob(s_blob, a.blob, a.blob_words, a.run_word, a.weight_word, a.pitch);
    for (int k = threadIdx.x; k < nk; k += blockDim.x) s_rv[k] = rvar_k[k];
    if (threadIdx.x < 4) s_s[cells + threadIdx.x] = 0xff;  // never below a scale: the masking leaves it

    float2 acc[Q];
#pragma unroll
    for (int i = 0; i < Q; i++) acc[i] = make_float2(0.0f, 0.0f);
    const FmaTap tap;

    for (int d = 0; d < a.D; d++) {
        __syncthreads();  // the tables staged; the previous direction's correlations are done
        // s*(d, .) and c_d = u / v_{d, s*}, u = g / den (0 outside the image), where the direction's
        // kernels reach; the other cells keep stale values that no correlation of this direction reads.
        // u is read again for every direction (from L2) instead of being kept in shared memory, which
        // leaves room for 128 x 64 tiles
        const uint8_t *plane = im.smap + static_cast<size_t>(d) * im.H * im.W;
        const float *rv_d = s_rv + d * a.S;
        const int4 dr = a.drect[d];
        for (int r = dr.x + warp; r < dr.y; r += nwarps) {
            const int gy = gy0 + r;
            const bool row_ok = gy >= 0 && gy < im.H;
            const size_t row = static_cast<size_t>(row_ok ? gy : 0);
            const uint8_t *prow = plane + row * im.W;
            const float *grow = im.g + row * im.g_pitch, *drow = im.rden + row * im.W;
            if (im.u_ready)
                build_field_row<true>(s_s, s_f, rv_d, prow, grow, drow, r * a.pitch, dr.z, dr.w, gx0, im.W, row_ok, lane);
            else
                build_field_row<false>(s_s, s_f, rv_d, prow, grow, drow, r * a.pitch, dr.z, dr.w, gx0, im.W, row_ok, lane);
        }
        __syncthreads();
        // telescoped scales: zero the field where s* < s, as far as D_s reaches, then correlate
        for (int s = 0; s < a.S; s++) {
            const int k = d * a.S + s;
            if (s > 0) {
                const int4 rc = a.rect[k];
                const unsigned below = 0x01010101u * static_cast<unsigned>(s);
                __syncthreads();  // every correlation of the previous scale is done with the field
                // every 4-cell word from the rectangle's first cell to its last, as one flat range over all
                // threads (the cells beside the rectangle in those rows are masked too: zeroing a cell with
                // s* < s anywhere keeps the field c_d [s* >= s]).  Per byte, (s* | 0x80) - s keeps its top
                // bit exactly where s* >= s (scales are below 0x80) and borrows from no other byte; cells
                // outside this direction's region hold stale bytes, which no correlation reads.
                const int w0 = (rc.x * a.pitch + rc.z) >> 2, w1 = ((rc.y - 1) * a.pitch + rc.w + 3) >> 2;
                const unsigned *sw = reinterpret_cast<const unsigned *>(s_s);
                for (int wi = w0 + static_cast<int>(threadIdx.x); wi < w1; wi += Shape::kThreads) {
                    const unsigned ge = ((sw[wi] | 0x80808080u) - below) & 0x80808080u;
                    if (ge != 0x80808080u) {  // a cell of the word has s* < s: keep the others
                        const unsigned keep = (ge >> 7) * 0xffu;  // 0xff per kept cell
                        float4 *f4 = reinterpret_cast<float4 *>(s_f) + wi;
                        float4 v = *f4;
                        v.x = __uint_as_float(__float_as_uint(v.x) & __byte_perm(keep, 0u, 0x0000));
                        v.y = __uint_as_float(__float_as_uint(v.y) & __byte_perm(keep, 0u, 0x1111));
                        v.z = __uint_as_float(__float_as_uint(v.z) & __byte_perm(keep, 0u, 0x2222));
                        v.w = __uint_as_float(__float_as_uint(v.w) & __byte_perm(keep, 0u, 0x3333));
                        *f4 = v;
                    }
                }
                __syncthreads();
            }
            const int r_end = s_blob[k + 1];
            for (int r = s_blob[k] + group; r < r_end; r += G) {
                const int4 run = s_runs[r];  // (field offset, len, float4 weight index): see stage_blob
                const int o = lane_off + run.x;
                conv_run<Q>(acc, PairWin{s_f + o, s_f + o + pair_rows}, s_wq + run.z, run.y, tap);
            }
        }
    }
    // groups 1, 2, ... hand their partial sums to group 0 in turn through the field (free after the
    // barrier); group 0 adds them in group order
    float2 *s_h = reinterpret_cast<float2 *>(s_f);
    for (int g = 1; g < G; g++) {
        __syncthreads();
        if (group == g) {
#pragma unroll
            for (int i = 0; i < Q; i++) s_h[i * Shape::kGroupThreads + gtid] = acc[i];
        }
        __syncthreads();
        if (group == 0) {
#pragma unroll
            for (int i = 0; i < Q; i++) {
                const float2 other = s_h[i * Shape::kGroupThreads + gtid];
                acc[i] = make_float2(acc[i].x + other.x, acc[i].y + other.y);
            }
        }
    }
    if (group == 0) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int oy = y0 + ty + kGatherPair * h;
            if (oy >= im.H) break;
            float *o = im.grad + static_cast<size_t>(oy) * im.grad_pitch + x0 + tx;
#pragma unroll
            for (int i = 0; i < Q; i++)
                if (x0 + tx + i < im.W) o[i] = h == 0 ? acc[i].x : acc[i].y;
        }
    }
}

// u = g * (1 / den) written over 1 / den, once per image between the two passes of the recomputing
// adjoints (the 1/den map is their own workspace there), so that the gather's per-direction field builds
// read one map instead of two.  The product is the one the gather forms otherwise.  Images blockIdx.y,
// blockIdx.y + gridDim.y, ... of a batched plan (images: n descriptors), else the single one.
__global__ void lpaici_adjoint_u_kernel(const GatherImage *images, const GatherImage single, int n) {
    for (int i = blockIdx.y; i < n; i += gridDim.y) {
        const GatherImage im = images ? images[i] : single;
        float *u = const_cast<float *>(im.rden);
        for (int y = blockIdx.x; y < im.H; y += gridDim.x) {
            const float *grow = im.g + static_cast<size_t>(y) * im.g_pitch;
            float *urow = u + static_cast<size_t>(y) * im.W;
            for (int x = threadIdx.x; x < im.W; x += blockDim.x) urow[x] = grow[x] * urow[x];
        }
    }
}

int u_launch(const GatherImage *images, const GatherImage &single, int n, int max_h, cudaStream_t stream) {
    const dim3 grid(static_cast<unsigned>(std::min(max_h, 1184)), static_cast<unsigned>(std::min(n, 65535)));
    lpaici_adjoint_u_kernel<<<grid, 256, 0, stream>>>(images, single, n);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "adjoint u launch");
}

}  // namespace

namespace {

// The gather kernel of tile height index I .. kGatherNWY - 1 whose WY is wy (null when none is).
template <int I>
const void *gather_fn(int wy) {
    if constexpr (I < kGatherNWY) {
        if (wy == kGatherWYs[I]) return reinterpret_cast<const void *>(lpaici_adjoint_gather_kernel<kGatherWYs[I]>);
        return gather_fn<I + 1>(wy);
    } else {
        return nullptr;
    }
}

template <int I>
bool gather_launch_at(const GatherArgs &ga, int wy, unsigned grid, size_t smem, cudaStream_t stream) {
    if constexpr (I < kGatherNWY) {
        constexpr int WY = kGatherWYs[I];
        if (wy != WY) return gather_launch_at<I + 1>(ga, wy, grid, smem, stream);
        lpaici_adjoint_gather_kernel<WY><<<grid, GatherShape<WY>::kThreads, smem, stream>>>(ga);
        return true;
    } else {
        return false;
    }
}

int gather_launch(const GatherArgs &ga, int wy, unsigned grid, size_t smem, cudaStream_t stream) {
    if (!gather_launch_at<0>(ga, wy, grid, smem, stream))
        return set_error(LPAICI_ERR_INVALID_ARG, "adjoint gather: no kernel for tile height %d", wy);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "adjoint gather launch");
}

// Chooses the tile height (*wy: 16 * wy output rows), fills the geometry and the per-kernel rectangles of
// the in-place masking; smem receives the dynamic shared memory, checked against the device.
int gather_setup(const lpaici_kernelset *ks, const int *adj_blob, GatherArgs *ga, size_t *smem, int *wy) {
    const BlobLayout &L = ks->adj_layout;
    const int nk = ks->D * ks->S;
    ga->R = ks->radius;
    ga->blob_words = L.total_words;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    *wy = 0;
    GatherGeom geo{};
    constexpr int kTW = GatherShape<1>::kTW;
    for (const int w : kGatherWYs) {
        geo = GatherGeom::make(kTW, GatherShape<1>::kTH * w, ga->R);
        *smem = gather_smem(L.total_words, nk, geo);
        if (*smem <= static_cast<size_t>(max_optin)) {
            *wy = w;
            break;
        }
    }
    if (*wy == 0)
        return set_error(LPAICI_ERR_UNSUPPORTED, "adjoint tile needs %zu B of shared memory, device allows %d", *smem,
                         max_optin);
    ga->th = GatherShape<1>::kTH * *wy;
    ga->pitch = geo.pitch;
    ga->rows = geo.rows;
    ga->D = ks->D;
    ga->S = ks->S;
    ga->blob = adj_blob;
    ga->run_word = L.run_word;
    ga->weight_word = L.weight_word;
    for (int k = 0; k < nk; k++) {
        // a lane reads rows ty + R + dy and ty + 8 + R + dy (ty + 8 < th) and columns
        // tx + R + dx0 + [0, len + Q - 1) (tx + Q <= tile width): rows [R + dy_min, R + th + dy_max),
        // columns [R + dx_min, R + tile width + dx_max)
        int ylo = 0, yhi = -1, xlo = 0, xhi = -1;
        for (int r = ks->adj_blob[k]; r < ks->adj_blob[k + 1]; r++) {
            const int *run = &ks->adj_blob[L.run_word + 4 * r];
            const int dy = run[0], c0 = run[1], c1 = run[1] + run[2] - 1;
            if (yhi < ylo) {
                ylo = yhi = dy;
                xlo = c0;
                xhi = c1;
            } else {
                ylo = std::min(ylo, dy);
                yhi = std::max(yhi, dy);
                xlo = std::min(xlo, c0);
                xhi = std::max(xhi, c1);
            }
        }
        if (yhi < ylo)
            ga->rect[k] = make_int4(0, 0, 0, 0);  // no taps
        else
            ga->rect[k] = make_int4(std::max(0, ga->R + ylo), std::min(geo.rows, ga->R + ga->th + yhi),
                                    std::max(0, ga->R + xlo), std::min(geo.pitch, ga->R + kTW + xhi));
    }
    for (int d = 0; d < ks->D; d++) {
        int4 u = make_int4(0, 0, 0, 0);
        for (int s = 0; s < ks->S; s++) {
            const int4 r = ga->rect[d * ks->S + s];
            if (r.y <= r.x || r.w <= r.z) continue;
            if (u.y <= u.x) {
                u = r;
            } else {
                u = make_int4(std::min(u.x, r.x), std::max(u.y, r.y), std::min(u.z, r.z), std::max(u.w, r.w));
            }
        }
        ga->drect[d] = u;
    }
    cudaError_t e = cudaFuncSetAttribute(gather_fn<0>(*wy), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(*smem));
    return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "adjoint gather attributes");
}

long gather_tiles(int width, int height, int th, int *tiles_x) {
    *tiles_x = (width + GatherShape<1>::kTW - 1) / GatherShape<1>::kTW;
    return static_cast<long>(*tiles_x) * ((height + th - 1) / th);
}

}  // namespace

int gather_pass(const lpaici_kernelset *ks, const int *adj_blob, const uint8_t *smap, const float *rden,
                const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch, int width, int height,
                float sigma, bool u_ready, cudaStream_t stream);

// The two passes over caller-provided storage (lpaici_backward, lpaici_backward_noalloc).
int adjoint_passes(const lpaici_kernelset *ks, const int *blob, const int *adj_blob, uint8_t *smap, float *rden,
                   const float *d_noisy, int noisy_pitch, const float *d_grad_out, int gout_pitch, float *d_grad_in,
                   int gin_pitch, int width, int height, float sigma, float gamma, cudaStream_t stream) {
    int tiles_x = 0;
    if (gather_tiles(width, height, 16, &tiles_x) > 0x7fffffffL)  // the shortest tile the gather may use
        return set_error(LPAICI_ERR_UNSUPPORTED, "image too large: %d x %d", width, height);

    // A. selection
    ImageArgs img{};
    img.in = d_noisy;
    img.out = nullptr;
    img.smap = smap;
    img.rden = rden;
    img.W = width;
    img.in_h = height;
    img.in_pitch = noisy_pitch;
    img.out_pitch = width;
    img.row_begin = 0;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    int rc = launch_forward(ks, img, tab, config_for(ks, width, height), stream);
    if (rc != LPAICI_OK) return rc;
    // u = g / den over the workspace's 1/den
    rc = u_launch(nullptr, GatherImage{d_grad_out, smap, rden, d_grad_in, nullptr, gout_pitch, gin_pitch, width, height, 0, 0},
                  1, height, stream);
    if (rc != LPAICI_OK) return rc;

    // B. gather
    return gather_pass(ks, adj_blob, smap, rden, d_grad_out, gout_pitch, d_grad_in, gin_pitch, width, height, sigma,
                       true, stream);
}

// Pass B alone, from the s* planes and 1/den of the image (pass A's outputs or a kept state), or u = g / den
// in place of 1/den (u_ready).
int gather_pass(const lpaici_kernelset *ks, const int *adj_blob, const uint8_t *smap, const float *rden,
                const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch, int width, int height,
                float sigma, bool u_ready, cudaStream_t stream) {
    GatherArgs ga{};
    size_t smem = 0;
    int wy = 0;
    int rc = gather_setup(ks, adj_blob, &ga, &smem, &wy);
    if (rc != LPAICI_OK) return rc;
    int tiles_x = 0;
    const long tiles = gather_tiles(width, height, ga.th, &tiles_x);
    if (tiles > 0x7fffffffL) return set_error(LPAICI_ERR_UNSUPPORTED, "image too large: %d x %d", width, height);
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, 1.0f, &tab);
    ga.single = GatherImage{d_grad_out, smap, rden, d_grad_in, nullptr, gout_pitch, gin_pitch, width, height, tiles_x,
                            u_ready ? 1 : 0};
    for (int k = 0; k < ks->D * ks->S; k++) ga.rvar[k] = 1.0f / tab.var[k];
    return gather_launch(ga, wy, static_cast<unsigned>(tiles), smem, stream);
}

namespace {

// The adjoint's workspace comes from a stream-ordered memory pool owned by this library, one per
// device, that keeps freed memory for the next call (release threshold: never).  The device's default
// pool returns memory to the driver at every synchronisation, so a caller that synchronises between
// calls would map the workspace afresh each time (about 20 bytes per pixel: tens of ms at 8192^2).
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_lock;
cudaMemPool_t g_pools[kMaxPoolDevices];

int workspace_pool(cudaMemPool_t *out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxPoolDevices)
        return set_error(LPAICI_ERR_UNSUPPORTED, "device %d beyond %d", dev, kMaxPoolDevices);
    std::lock_guard<std::mutex> hold(g_pool_lock);
    if (!g_pools[dev]) {
        int supported = 0;
        cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev);
        if (!supported)
            return set_error(LPAICI_ERR_UNSUPPORTED,
                             "device %d has no stream-ordered memory pools: use lpaici_backward_noalloc", dev);
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemPoolCreate(adjoint workspace)");
        uint64_t keep = ~uint64_t(0);
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return cuda_error(e, "cudaMemPoolSetAttribute(adjoint workspace)");
        }
        g_pools[dev] = pool;
    }
    *out = g_pools[dev];
    return LPAICI_OK;
}

}  // namespace

int check_adjoint_params(const lpaici_kernelset *ks, float sigma, const float *gamma, const char *who) {
    if (!(sigma > 0.0f) || !std::isfinite(sigma) || (gamma && (!(*gamma > 0.0f) || !std::isfinite(*gamma))))
        return set_error(LPAICI_ERR_INVALID_ARG, "%s: sigma and gamma need finite positive numbers", who);
    if (ks->S > kMaxScales)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%s: %d scales per direction; the adjoint supports at most %d", who,
                         ks->S, kMaxScales);
    return LPAICI_OK;
}

}  // namespace lpaici

using namespace lpaici;

extern "C" int lpaici_trim_workspace(void) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> hold(g_pool_lock);
        if (dev >= 0 && dev < kMaxPoolDevices) pool = g_pools[dev];
    }
    if (!pool) return LPAICI_OK;
    e = cudaMemPoolTrimTo(pool, 0);
    return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "cudaMemPoolTrimTo(adjoint workspace)");
}

extern "C" int lpaici_backward(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch,
                               const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch, int width,
                               int height, float sigma, float gamma, lpaici_stream_t stream_) {
    if (!ks || !d_noisy || !d_grad_out || !d_grad_in)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward: null argument");
    if (width <= 0 || height <= 0 || noisy_pitch < width || gout_pitch < width || gin_pitch < width)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward: bad size or pitch");
    int rc = check_adjoint_params(ks, sigma, &gamma, "lpaici_backward");
    if (rc != LPAICI_OK) return rc;
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const int *blob = nullptr, *adj = nullptr;
    rc = device_blob(ks, &blob);
    if (rc == LPAICI_OK) rc = device_adj_blob(ks, &adj);
    if (rc != LPAICI_OK) return rc;

    // transient workspace: D selection planes (bytes) and 1/den (floats)
    cudaMemPool_t pool = nullptr;
    rc = workspace_pool(&pool);
    if (rc != LPAICI_OK) return rc;
    const size_t npx = static_cast<size_t>(width) * height;
    void *ws = nullptr;
    const size_t smap_bytes = (static_cast<size_t>(ks->D) * npx + 255) & ~size_t(255);
    cudaError_t e = cudaMallocFromPoolAsync(&ws, smap_bytes + sizeof(float) * npx, pool, stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocFromPoolAsync(adjoint workspace)");
    uint8_t *smap = static_cast<uint8_t *>(ws);
    float *rden = reinterpret_cast<float *>(static_cast<char *>(ws) + smap_bytes);
    rc = adjoint_passes(ks, blob, adj, smap, rden, d_noisy, noisy_pitch, d_grad_out, gout_pitch, d_grad_in, gin_pitch,
                        width, height, sigma, gamma, stream);
    cudaError_t ef = cudaFreeAsync(ws, stream);
    if (rc == LPAICI_OK && ef != cudaSuccess) rc = cuda_error(ef, "cudaFreeAsync(adjoint workspace)");
    return rc;
}

// ---------------------------------------------------------------------------------------------
// Batched adjoint plan.
// ---------------------------------------------------------------------------------------------
struct lpaici_backward_batch {
    int device = -1;
    lpaici_batch *select = nullptr;  // pass A: the forward batch plan (out = null, s* and 1/den on)
    void *dev_mem = nullptr;         // s* planes | 1/den maps | GatherImage[n] | 1/v tables | items
    GatherArgs ga{};
    size_t smem = 0;
    int wy = 0;
    unsigned grid = 0;
    int n = 0, max_h = 0;  // images; the tallest one's rows (the u launch)
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

int backward_batch_enqueue(lpaici_backward_batch *b, cudaStream_t stream) {
    int rc = batch_plan_enqueue(b->select, stream);
    if (rc != LPAICI_OK) return rc;
    rc = u_launch(b->ga.images, GatherImage{}, b->n, b->max_h, stream);
    if (rc != LPAICI_OK) return rc;
    return gather_launch(b->ga, b->wy, b->grid, b->smem, stream);
}

void backward_batch_free(lpaici_backward_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    batch_plan_free(b->select);
    if (b->dev_mem) cudaFree(b->dev_mem);
    delete b;
}

size_t align256(size_t n) { return (n + 255) & ~size_t(255); }

}  // namespace

extern "C" int lpaici_backward_batch_create(const lpaici_kernelset *ks, const lpaici_grad_image *images, int n,
                                            const lpaici_batch_options *opts, lpaici_stream_t stream_,
                                            lpaici_backward_batch **out) {
    if (!ks || !images || n <= 0 || !out)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward_batch_create: bad argument");
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        const lpaici_grad_image &im = images[i];
        if (!im.noisy || !im.grad_out || !im.grad_in || im.width <= 0 || im.height <= 0 || im.noisy_pitch < im.width ||
            im.gout_pitch < im.width || im.gin_pitch < im.width)
            return set_error(LPAICI_ERR_INVALID_ARG, "adjoint batch image %d: bad pointer, size or pitch", i);
        const int rc = check_adjoint_params(ks, im.sigma, &im.gamma, "lpaici_backward_batch_create");
        if (rc != LPAICI_OK) return rc;
    }
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const int *adj = nullptr;
    int rc = device_adj_blob(ks, &adj);
    if (rc != LPAICI_OK) return rc;
    auto *b = new lpaici_backward_batch();
    cudaGetDevice(&b->device);
    rc = gather_setup(ks, adj, &b->ga, &b->smem, &b->wy);
    if (rc != LPAICI_OK) {
        backward_batch_free(b);
        return rc;
    }

    // plan memory: per image s* planes and 1/den, then the gather's descriptors, tables and items
    const int nk = ks->D * ks->S;
    std::vector<size_t> smap_off(n), rden_off(n);
    std::vector<int> tiles_x(n);
    size_t off = 0;
    long total_tiles = 0;
    for (int i = 0; i < n; i++) {
        const size_t npx = static_cast<size_t>(images[i].width) * images[i].height;
        smap_off[i] = off;
        off = align256(off + static_cast<size_t>(ks->D) * npx);
        rden_off[i] = off;
        off = align256(off + sizeof(float) * npx);
        total_tiles += gather_tiles(images[i].width, images[i].height, b->ga.th, &tiles_x[i]);
    }
    if (total_tiles > 0x7fffffffL) {
        backward_batch_free(b);
        return set_error(LPAICI_ERR_UNSUPPORTED, "adjoint batch too large: %ld tiles", total_tiles);
    }
    const size_t desc_off = off;
    off = align256(off + sizeof(GatherImage) * n);
    const size_t rvar_off = off;
    off = align256(off + sizeof(float) * static_cast<size_t>(n) * nk);
    const size_t item_off = off;
    off = align256(off + sizeof(int2) * static_cast<size_t>(total_tiles));
    cudaError_t e = cudaMalloc(&b->dev_mem, off);
    if (e != cudaSuccess) {
        backward_batch_free(b);
        return cuda_error(e, "cudaMalloc(adjoint batch plan)");
    }
    char *base = static_cast<char *>(b->dev_mem);
    std::vector<GatherImage> desc(n);
    std::vector<float> rvar(static_cast<size_t>(n) * nk);
    std::vector<int2> items;
    items.reserve(static_cast<size_t>(total_tiles));
    std::vector<BatchSpec> specs(n);
    for (int i = 0; i < n; i++) {
        const lpaici_grad_image &im = images[i];
        uint8_t *smap = reinterpret_cast<uint8_t *>(base + smap_off[i]);
        float *rden = reinterpret_cast<float *>(base + rden_off[i]);
        KernelTables tab;
        fill_tables(ks, nullptr, im.sigma, im.gamma, &tab);
        float *rv = rvar.data() + static_cast<size_t>(i) * nk;
        for (int k = 0; k < nk; k++) rv[k] = 1.0f / tab.var[k];
        desc[i] = GatherImage{im.grad_out, smap, rden, im.grad_in,
                              reinterpret_cast<const float *>(base + rvar_off) + static_cast<size_t>(i) * nk,
                              im.gout_pitch, im.gin_pitch, im.width, im.height, tiles_x[i], 1};
        b->max_h = std::max(b->max_h, im.height);
        int tx = 0;
        const long t = gather_tiles(im.width, im.height, b->ga.th, &tx);
        for (long j = 0; j < t; j++) items.push_back(make_int2(i, static_cast<int>(j)));
        specs[i] = BatchSpec{im.noisy, nullptr, smap, rden, im.width, im.height, im.noisy_pitch, im.width, im.sigma,
                             im.gamma};
    }
    e = cudaMemcpy(base + desc_off, desc.data(), sizeof(GatherImage) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + rvar_off, rvar.data(), sizeof(float) * rvar.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + item_off, items.data(), sizeof(int2) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        backward_batch_free(b);
        return cuda_error(e, "cudaMemcpy(adjoint batch plan)");
    }
    b->ga.images = reinterpret_cast<const GatherImage *>(base + desc_off);
    b->ga.items = reinterpret_cast<const int2 *>(base + item_off);
    b->grid = static_cast<unsigned>(total_tiles);
    b->n = n;

    int config = opts ? opts->tile_config : -1;
    if (config < 0) {
        std::vector<int> w(n), h(n);
        for (int i = 0; i < n; i++) {
            w[i] = specs[i].width;
            h[i] = specs[i].height;
        }
        config = config_for_images(ks, w.data(), h.data(), n);
    }
    rc = batch_plan_create(ks, specs.data(), n, config, false, stream, &b->select);
    if (rc != LPAICI_OK) {
        backward_batch_free(b);
        return rc;
    }
    b->use_graph = opts && opts->use_graph;
    if (b->use_graph) {
        cudaStream_t cap = nullptr;
        e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = backward_batch_enqueue(b, cap);
            const cudaError_t e2 = cudaStreamEndCapture(cap, &b->graph);
            if (rc == LPAICI_OK && e2 != cudaSuccess) rc = cuda_error(e2, "cudaStreamEndCapture");
            if (rc == LPAICI_OK) {
                e = cudaGraphInstantiate(&b->exec, b->graph, 0);
                if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphInstantiate");
            }
        } else {
            rc = cuda_error(e, "graph capture");
        }
        if (cap) cudaStreamDestroy(cap);
        if (rc == LPAICI_OK) {
            e = cudaGraphUpload(b->exec, stream);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphUpload");
        }
        if (rc != LPAICI_OK) {
            backward_batch_free(b);
            return rc;
        }
    }
    *out = b;
    return LPAICI_OK;
}

extern "C" int lpaici_backward_batch_run(lpaici_backward_batch *b, lpaici_stream_t stream_) {
    if (!b) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward_batch_run: null plan");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != b->device)
        return set_error(LPAICI_ERR_INVALID_ARG, "adjoint batch planned on device %d, current device is %d", b->device,
                         dev);
    if (b->use_graph) {
        const cudaError_t e = cudaGraphLaunch(b->exec, stream);
        return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "cudaGraphLaunch");
    }
    return backward_batch_enqueue(b, stream);
}

extern "C" int lpaici_backward_batch_destroy(lpaici_backward_batch *b) {
    if (b) {
        int cur = -1;
        cudaGetDevice(&cur);
        cudaSetDevice(b->device);
        cudaDeviceSynchronize();
        backward_batch_free(b);
        if (cur >= 0) cudaSetDevice(cur);
    }
    return LPAICI_OK;
}

// ---------------------------------------------------------------------------------------------
// Kept state: the forward stores what its adjoint needs, the adjoint runs the gather only.
// ---------------------------------------------------------------------------------------------
namespace {

size_t state_smap_bytes(const lpaici_kernelset *ks, int width, int height) {
    return (static_cast<size_t>(ks->D) * width * height + 255) & ~size_t(255);
}

int state_args(const lpaici_kernelset *ks, int width, int height, float sigma, const char *who) {
    if (!ks) return set_error(LPAICI_ERR_INVALID_ARG, "%s: null kernel set", who);
    if (width <= 0 || height <= 0) return set_error(LPAICI_ERR_INVALID_ARG, "%s: bad size %d x %d", who, width, height);
    return check_adjoint_params(ks, sigma, nullptr, who);
}

}  // namespace

extern "C" size_t lpaici_adjoint_state_bytes(const lpaici_kernelset *ks, int width, int height) {
    if (!ks || width <= 0 || height <= 0) return 0;
    return state_smap_bytes(ks, width, height) + sizeof(float) * static_cast<size_t>(width) * height;
}

extern "C" int lpaici_forward_state(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch,
                                    float *d_denoised, int out_pitch, int width, int height, float sigma, float gamma,
                                    void *d_state, lpaici_stream_t stream_) {
    int rc = state_args(ks, width, height, sigma, "lpaici_forward_state");
    if (rc != LPAICI_OK) return rc;
    if (!d_noisy || !d_denoised || !d_state || noisy_pitch < width || out_pitch < width)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_forward_state: null pointer or bad pitch");
    rc = check_adjoint_params(ks, sigma, &gamma, "lpaici_forward_state");
    if (rc != LPAICI_OK) return rc;
    const int *blob = nullptr;
    rc = device_blob(ks, &blob);
    if (rc != LPAICI_OK) return rc;
    ImageArgs img{};
    img.in = d_noisy;
    img.out = d_denoised;
    img.smap = static_cast<uint8_t *>(d_state);
    img.rden = reinterpret_cast<float *>(static_cast<char *>(d_state) + state_smap_bytes(ks, width, height));
    img.W = width;
    img.in_h = height;
    img.in_pitch = noisy_pitch;
    img.out_pitch = out_pitch;
    img.row_begin = 0;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    return launch_forward(ks, img, tab, config_for(ks, width, height), reinterpret_cast<cudaStream_t>(stream_));
}

extern "C" int lpaici_backward_state(const lpaici_kernelset *ks, const void *d_state, const float *d_grad_out,
                                     int gout_pitch, float *d_grad_in, int gin_pitch, int width, int height, float sigma,
                                     lpaici_stream_t stream_) {
    int rc = state_args(ks, width, height, sigma, "lpaici_backward_state");
    if (rc != LPAICI_OK) return rc;
    if (!d_state || !d_grad_out || !d_grad_in || gout_pitch < width || gin_pitch < width)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward_state: null pointer or bad pitch");
    const int *adj = nullptr;
    rc = device_adj_blob(ks, &adj);
    if (rc != LPAICI_OK) return rc;
    const uint8_t *smap = static_cast<const uint8_t *>(d_state);
    const float *rden =
        reinterpret_cast<const float *>(static_cast<const char *>(d_state) + state_smap_bytes(ks, width, height));
    return gather_pass(ks, adj, smap, rden, d_grad_out, gout_pitch, d_grad_in, gin_pitch, width, height, sigma,
                       false, reinterpret_cast<cudaStream_t>(stream_));
}
