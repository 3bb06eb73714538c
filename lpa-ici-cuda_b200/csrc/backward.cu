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
//      window of P partial outputs: P FMAs per weight, one shared-memory atomic per finished output;
//   3. write-back: the gradient tile is added to the output with global atomics (halos of
//      neighbouring tiles overlap).
// No counterpart in the reference.
#include "configs.h"
#include "tile_core.cuh"

namespace lpaici {

// dst[m] += sum_{i + j = m} c[i] * w[j], m < len + P - 1; window slot m % P holds output m.
template <int P>
__device__ __forceinline__ void scatter_run(const float (&c)[P], float *dst, const float *__restrict__ w, int len) {
    float acc[P];
#pragma unroll
    for (int i = 0; i < P; i++) acc[i] = 0.0f;
    const int n_out = len + P - 1;
    for (int j0 = 0; j0 < n_out; j0 += P) {
#pragma unroll
        for (int q = 0; q < P; q++) {
            const int j = j0 + q;
            if (j < len) {
                const float wt = w[j];
#pragma unroll
                for (int i = 0; i < P; i++) acc[(i + q) % P] = fmaf(c[i], wt, acc[(i + q) % P]);
            }
            if (j < n_out) {
                atomicAdd(dst + j, acc[q]);  // output j is complete
                acc[q] = 0.0f;
            }
        }
    }
}

template <int P, int WX, int WY>
__global__ void __launch_bounds__(32 * WX * WY)
    lpaici_backward_kernel(const __grid_constant__ ImageArgs img, const __grid_constant__ KernelTables tab) {
    using Shape = TileShape<P, WX, WY>;
    extern __shared__ __align__(16) int smem[];
    const int D = tab.D, S = tab.S, R = tab.R, nk = D * S;
    const int tab_words = (2 * nk + 3) & ~3;
    int *s_blob = smem;
    float *s_var = reinterpret_cast<float *>(smem + tab.blob_words);
    float *s_thr = s_var + nk;
    float *s_tile = reinterpret_cast<float *>(smem + tab.blob_words + tab_words);
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, R);
    const int x0 = blockIdx.x * Shape::kTileW, y0 = blockIdx.y * Shape::kTileH;

    stage_words(s_blob, tab.blob, tab.blob_words);
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
        s_var[i] = tab.var[i];
        s_thr[i] = tab.thr[i];
    }
    load_tile(s_tile, img, x0, y0, R, g);
    __syncthreads();

    const LaneGeom<P, WX> lg;
    const int oy = y0 + lg.ty, ox = x0 + lg.tx;
    unsigned valid = 0;
    if (oy < img.rows_out) {
#pragma unroll
        for (int i = 0; i < P; i++)
            if (ox + i < img.W) valid |= 1u << i;
    }
    const int lane_off = (lg.ty + R) * g.pitch + lg.tx + g.HL;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + tab.run_word);
    const float *s_w = reinterpret_cast<const float *>(s_blob + tab.weight_word);

    // phase 1: selection of every direction, sum of the weights 1/v
    unsigned long long sel[P];
    float den[P];
#pragma unroll
    for (int i = 0; i < P; i++) {
        sel[i] = 0ull;
        den[i] = 0.0f;
    }
    for (int d = 0; d < D; d++) {
        float best[P], bvar[P];
        int sidx[P];
        direction_sweep<P>(d, S, valid, s_tile + lane_off, g.pitch, s_blob, s_runs, s_w, s_var, s_thr, best, bvar,
                           sidx);
#pragma unroll
        for (int i = 0; i < P; i++) {
            sel[i] |= static_cast<unsigned long long>(sidx[i]) << (4 * d);
            den[i] = __fadd_rn(den[i], __fdiv_rn(1.0f, bvar[i]));
        }
    }
    __syncthreads();  // done reading the input tile

    // phase 2: the tile becomes the gradient accumulator
    for (int i = threadIdx.x; i < g.rows * g.pitch; i += blockDim.x) s_tile[i] = 0.0f;
    float gp[P];
    const float *gsrc = img.gout + static_cast<size_t>(oy) * img.gout_pitch + ox;
#pragma unroll
    for (int i = 0; i < P; i++) gp[i] = (valid & (1u << i)) ? __ldg(gsrc + i) : 0.0f;
    __syncthreads();

    float *lane_grad = s_tile + lane_off;
    for (int d = 0; d < D; d++) {
        float c[P];
        unsigned present = 0;
#pragma unroll
        for (int i = 0; i < P; i++) {
            const int s = static_cast<int>((sel[i] >> (4 * d)) & 15ull);
            const float v = s_var[d * S + s];
            c[i] = (valid & (1u << i)) ? gp[i] * ((1.0f / v) / den[i]) : 0.0f;
            if (valid & (1u << i)) present |= 1u << s;
        }
        present = __reduce_or_sync(0xffffffffu, present);
        while (present) {
            const int s = __ffs(present) - 1;
            present &= present - 1;
            float cs[P];
#pragma unroll
            for (int i = 0; i < P; i++) cs[i] = (static_cast<int>((sel[i] >> (4 * d)) & 15ull) == s) ? c[i] : 0.0f;
            const int k = d * S + s;
            const int rb = s_blob[k], re = s_blob[k + 1];
            for (int r = rb; r < re; r++) {
                const int4 run = s_runs[r];
                scatter_run<P>(cs, lane_grad + run.x * g.pitch + run.y, s_w + run.w, run.z);
            }
        }
    }
    __syncthreads();

    // phase 3: add the gradient tile (with its halo) to the output
    const int gy0 = y0 + img.row_begin - R, gx0 = x0 - g.HL;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int r = warp; r < g.rows; r += nwarps) {
        const int gy = gy0 + r;
        if (gy < 0 || gy >= img.in_h) continue;
        float *dst = img.out + static_cast<size_t>(gy) * img.out_pitch;
        const float *src = s_tile + r * g.pitch;
        for (int cc = lane; cc < g.pitch; cc += 32) {
            const int gx = gx0 + cc;
            if (gx >= 0 && gx < img.W) {
                const float v = src[cc];
                if (v != 0.0f) atomicAdd(dst + gx, v);
            }
        }
    }
}

namespace {

template <int P, int WX, int WY>
int launch_bwd(const ImageArgs &img, const KernelTables &tab, cudaStream_t stream) {
    using Shape = TileShape<P, WX, WY>;
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R);
    const int nk = tab.D * tab.S;
    const size_t smem = sizeof(int) * (tab.blob_words + ((2 * nk + 3) & ~3)) + sizeof(float) * g.pitch * g.rows;
    auto kern = lpaici_backward_kernel<P, WX, WY>;
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

int launch_backward(const lpaici_kernelset *ks, const ImageArgs &img, const KernelTables &tab, cudaStream_t stream) {
    (void)ks;
    return launch_bwd<9, 2, 4>(img, tab, stream);
}

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
    return launch_backward(ks, img, tab, stream);
}
