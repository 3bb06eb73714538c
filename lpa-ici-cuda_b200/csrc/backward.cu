// backward.cu -- adjoint of the LPA-ICI forward with the ICI selection held fixed.
//
// For L = sum_p g[p] * out[p] and the selected scale s*(d,p) of every direction and pixel frozen,
// out is linear in the input x:  out(p) = sum_d alpha_d(p) * sum_t h_{d,s*}(t) x(p + t - c), with
// alpha_d(p) = (1/v_d(p)) / sum_d' (1/v_d'(p)).  Hence
//     dL/dx(q) = sum_d sum_p g(p) * alpha_d(p) * h_{d,s*(d,p)}(q - p + c)      (zero padding).
// One CTA per output tile, in three phases:
//   1. recompute: the forward's exact ICI sweep over the input tile yields s*(d,p) for all 16
//      directions (packed 4 bits per direction) and sum_d 1/v_d -- no scale map is stored or read;
//   2. scatter: the input tile's shared memory becomes a gradient tile (tile + halo R); for every
//      direction and every scale present in the warp, each thread spreads c_i = g_i * alpha_{d,i}
//      (zero for pixels that selected another scale) through the kernel's row runs with a sliding
//      window of 4 partial outputs per pixel row: 4 FMAs per weight, one shared-memory atomic per
//      finished output;
//   3. write-back: the gradient tile is added to the output with global atomics (halos of
//      neighbouring tiles overlap).
// No counterpart in the reference.
#include "configs.h"
#include "tile_core.cuh"

namespace lpaici {

// dst[j] += sum_{i + k = j} c[i] * w_k for j < len + 3: the transpose of conv_run for one pixel row.
// A window of 4 partial outputs slides along the run (slot j % 4 holds output j); every finished
// output is added to shared memory with one atomic.  wq holds the run's duplicated weights.
__device__ __forceinline__ void scatter_run(const float (&c)[4], float *dst, const float4 *__restrict__ wq, int len) {
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const int n_out = len + 3;
    for (int j0 = 0; j0 < n_out; j0 += 4) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int j = j0 + q;
            if (j < len) {  // taps of the run only (its weights are padded to an even count)
                const float4 wp = wq[j >> 1];
                const float w = (q & 1) ? wp.z : wp.x;
#pragma unroll
                for (int i = 0; i < 4; i++) acc[(i + q) & 3] = fmaf(c[i], w, acc[(i + q) & 3]);
            }
            if (j < n_out) {
                atomicAdd(dst + j, acc[q]);
                acc[q] = 0.0f;
            }
        }
    }
}

template <int WX, int WY>
__global__ void __launch_bounds__(32 * WX * WY, 1)
    lpaici_backward_kernel(const __grid_constant__ ImageArgs img, const __grid_constant__ KernelTables tab) {
    using Shape = TileShape<WX, WY>;
    extern __shared__ __align__(16) int smem[];
    const int D = tab.D, S = tab.S, nk = D * S;
    int *s_blob = smem;
    float *s_tab = reinterpret_cast<float *>(smem + tab.blob_words);
    float2 *s_tile = reinterpret_cast<float2 *>(smem + tab.blob_words + table_words(nk));
    float *s_grad = reinterpret_cast<float *>(s_tile);  // phase 2 reuses the tile's memory
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R);
    const int R = g.R, gpitch = g.pitch2, grows = Shape::kTileH + 2 * R;
    const int x0 = blockIdx.x * Shape::kTileW, y0 = blockIdx.y * Shape::kTileH;

    stage_words(s_blob, tab.blob, tab.blob_words);
    stage_tables(s_tab, tab.var, tab.thr, nk);
    load_tile(s_tile, img, x0, y0, g);
    __syncthreads();

    const LaneGeom<WX> lg;
    const int oy = y0 + lg.ty, ox = x0 + lg.tx;
    unsigned valid = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
        if (oy + 8 * (i & 1) < img.rows_out && ox + (i >> 1) < img.W) valid |= 1u << i;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + tab.run_word);
    const float4 *s_wq = reinterpret_cast<const float4 *>(s_blob + tab.weight_word);
    const float *s_thr = s_tab + nk, *s_rvar = s_tab + 2 * nk;

    // phase 1: the selection of every direction (4 bits each) and sum_d 1/v_d, per pixel
    unsigned long long sel[8];
    float den[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        sel[i] = 0ull;
        den[i] = 0.0f;
    }
    const float2 *lane_tile = s_tile + (lg.ty + R) * g.pitch2 + lg.tx + R;
    for (int d = 0; d < D; d++) {
        float best[8];
        unsigned sidx;
        direction_sweep(d, S, valid, lane_tile, g.pitch2, s_blob, s_runs, s_wq, s_thr,
                        make_float2(tab.neg_zero, tab.neg_zero), best, sidx);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const unsigned si = (sidx >> (4 * i)) & 15u;
            sel[i] |= static_cast<unsigned long long>(si) << (4 * d);
            den[i] += s_rvar[d * S + si];
        }
    }
    __syncthreads();  // done reading the input tile

    // phase 2: the tile's memory becomes the gradient accumulator (tile + R halo, plain floats)
    for (int i = threadIdx.x; i < grows * gpitch; i += blockDim.x) s_grad[i] = 0.0f;
    float gp[8];
#pragma unroll
    for (int i = 0; i < 8; i++)
        gp[i] = (valid & (1u << i)) ? __ldg(img.gout + static_cast<size_t>(oy + 8 * (i & 1)) * img.gout_pitch + ox +
                                            (i >> 1))
                                    : 0.0f;
    __syncthreads();

    float *lane_grad = s_grad + (lg.ty + R) * gpitch + lg.tx + R;
    for (int d = 0; d < D; d++) {
        float c[8];
        unsigned present = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int s = static_cast<int>((sel[i] >> (4 * d)) & 15ull);
            c[i] = (valid & (1u << i)) ? gp[i] * (s_rvar[d * S + s] / den[i]) : 0.0f;
            if (valid & (1u << i)) present |= 1u << s;
        }
        present = __reduce_or_sync(0xffffffffu, present);
        while (present) {
            const int s = __ffs(present) - 1;
            present &= present - 1;
            float c0[4], c1[4];  // rows ty and ty + 8
#pragma unroll
            for (int m = 0; m < 4; m++) {
                c0[m] = (static_cast<int>((sel[2 * m] >> (4 * d)) & 15ull) == s) ? c[2 * m] : 0.0f;
                c1[m] = (static_cast<int>((sel[2 * m + 1] >> (4 * d)) & 15ull) == s) ? c[2 * m + 1] : 0.0f;
            }
            const int k = d * S + s;
            const int rb = s_blob[k], re = s_blob[k + 1];
            for (int r = rb; r < re; r++) {
                const int4 run = s_runs[r];
                float *dst = lane_grad + run.x * gpitch + run.y;
                scatter_run(c0, dst, s_wq + (run.w >> 1), run.z);
                scatter_run(c1, dst + 8 * gpitch, s_wq + (run.w >> 1), run.z);
            }
        }
    }
    __syncthreads();

    // phase 3: add the gradient tile (with its halo) to the output
    const int gy0 = y0 + img.row_begin - R, gx0 = x0 - R;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < grows; r += nwarps) {
        const int gy = gy0 + r;
        if (gy < 0 || gy >= img.in_h) continue;
        float *dst = img.out + static_cast<size_t>(gy) * img.out_pitch;
        const float *src = s_grad + r * gpitch;
        for (int cc = lane; cc < gpitch; cc += 32) {
            const int gx = gx0 + cc;
            if (gx >= 0 && gx < img.W) {
                const float v = src[cc];
                if (v != 0.0f) atomicAdd(dst + gx, v);
            }
        }
    }
}

namespace {

template <int WX, int WY>
int launch_bwd(const ImageArgs &img, const KernelTables &tab, cudaStream_t stream) {
    using Shape = TileShape<WX, WY>;
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R);
    const int nk = tab.D * tab.S;
    const size_t grad_bytes = sizeof(float) * static_cast<size_t>(g.pitch2) * (Shape::kTileH + 2 * tab.R);
    const size_t region = g.tile_bytes() > grad_bytes ? g.tile_bytes() : grad_bytes;
    const size_t smem = sizeof(int) * (tab.blob_words + table_words(nk)) + region;
    auto kern = lpaici_backward_kernel<WX, WY>;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > static_cast<size_t>(max_optin))
        return set_error(LPAICI_ERR_UNSUPPORTED, "backward tile needs %zu B of shared memory, device allows %d", smem,
                         max_optin);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(backward)");
    const dim3 grid((img.W + Shape::kTileW - 1) / Shape::kTileW, (img.rows_out + Shape::kTileH - 1) / Shape::kTileH);
    if (grid.y > 65535u) return set_error(LPAICI_ERR_UNSUPPORTED, "image too tall: %d rows", img.rows_out);
    kern<<<grid, Shape::kThreads, smem, stream>>>(img, tab);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "backward launch");
    return LPAICI_OK;
}

}  // namespace

#define LPAICI_BWD_CASE(idx, WX, WY) \
    case idx: return launch_bwd<WX, WY>(img, tab, stream);

int launch_backward(const lpaici_kernelset *ks, const ImageArgs &img, const KernelTables &tab, int config,
                    cudaStream_t stream) {
    (void)ks;
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_BWD_CASE)
        default: return set_error(LPAICI_ERR_INVALID_ARG, "tile config %d out of range", config);
    }
}
#undef LPAICI_BWD_CASE

}  // namespace lpaici

using namespace lpaici;

extern "C" int lpaici_backward(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch,
                               const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch, int width,
                               int height, float sigma, float gamma, lpaici_stream_t stream_) {
    if (!ks || !d_noisy || !d_grad_out || !d_grad_in)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward: null argument");
    if (width <= 0 || height <= 0 || noisy_pitch < width || gout_pitch < width || gin_pitch < width)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward: bad size or pitch");
    if (!(sigma > 0.0f) || !(gamma > 0.0f))
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward: sigma and gamma need positive numbers");
    if (ks->D > 16 || ks->S > 16)
        return set_error(LPAICI_ERR_UNSUPPORTED, "lpaici_backward supports at most 16 directions and 16 scales");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const int *blob = nullptr;
    int rc = device_blob(ks, &blob);
    if (rc != LPAICI_OK) return rc;
    cudaError_t e = cudaMemset2DAsync(d_grad_in, sizeof(float) * gin_pitch, 0, sizeof(float) * width, height, stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMemset2DAsync(grad)");
    ImageArgs img{};
    img.in = d_noisy;
    img.out = d_grad_in;
    img.gout = d_grad_out;
    img.smap = nullptr;
    img.W = width;
    img.in_h = height;
    img.in_pitch = noisy_pitch;
    img.out_pitch = gin_pitch;
    img.gout_pitch = gout_pitch;
    img.row_begin = 0;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    return launch_backward(ks, img, tab, default_config(ks), stream);
}
