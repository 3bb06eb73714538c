// backward.cu -- adjoint of the LPA-ICI forward with the ICI selection held fixed.
//
// For L = sum_p g[p] * out[p] and the selected scale s*(d,p) of every direction and pixel frozen,
// out is linear in the input x:  out(p) = sum_d alpha_d(p) * sum_t h_{d,s*}(t) x(p + t - c), with
// alpha_d(p) = (1/v_d(p)) / den(p), den(p) = sum_d' 1/v_d'(p).  Hence, with c_d(p) = g(p) alpha_d(p),
//     dL/dx(q) = sum_d sum_s sum_t h_{d,s}(t) [s*(d, q - t + c) = s] c_d(q - t + c)        (zero padding)
// i.e. for every direction and scale, a correlation of the masked field c_d [s* = s] with the kernel
// mirrored through its centre.  Two launches:
//   A. selection: the forward's exact tile sweep recomputes s*(d,p) (one byte per direction and
//      pixel) and den(p) into a transient workspace -- the forward stores nothing for the adjoint;
//   B. gather: one CTA per output tile builds, per direction, c_d and s* on the tile plus its R-pixel
//      halo in shared memory; per scale present there it masks the field and correlates it with the
//      mirrored kernel's row runs (register sliding window, 9 outputs per thread, FFMA -- the adjoint
//      is checked against FP64 finite differences, not bit patterns).  Every output is written once:
//      no atomics, deterministic.
// No counterpart in the reference.
#include "configs.h"
#include "tile_core.cuh"

namespace lpaici {

namespace {

constexpr int kGatherP = 9;  // outputs per thread (odd: conflict-free scalar shared loads)
constexpr int kGatherWX = 2, kGatherWY = 8;
constexpr int kGatherTW = kGatherWX * 4 * kGatherP, kGatherTH = kGatherWY * 8;  // 72 x 64, 512 threads

struct GatherArgs {
    const float *g;        // cotangent, pitch g_pitch
    const uint8_t *smap;   // D x H x W selected scales (pass A)
    const float *den;      // H x W, pitch W (pass A)
    float *grad;           // result, pitch grad_pitch
    int g_pitch, grad_pitch, W, H;
    int D, S, R;
    const int *blob;       // mirrored kernels (lpaici_kernelset::adj_blob)
    int blob_words, run_word, weight_word;
    int pitch, rows;       // shared-memory field geometry (floats)
    float rvar[kMaxKernels];
};

// Smallest pitch >= need with (pitch / 4) odd: scalar loads of 8 rows x 4 column groups of 9 hit 32
// different banks.
__host__ __device__ inline int field_pitch(int need) {
    int p = (need + 3) & ~3;
    if (((p >> 2) & 1) == 0) p += 4;
    return p;
}

// acc[i] += sum_{j < len} w[j] * src[i + j] for the thread's P outputs (sliding window, FFMA).
template <int P>
__device__ __forceinline__ void gather_run(float (&acc)[P], const float *__restrict__ src, const float *__restrict__ w,
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
            for (int i = 0; i < P; i++) acc[i] = fmaf(wt, win[(j + i) % P], acc[i]);
        }
    }
#pragma unroll
    for (int j = 0; j < P - 1; j++) {
        if (k + j < len) {
            win[(j + P - 1) % P] = src[k + j + P - 1];
            const float wt = w[k + j];
#pragma unroll
            for (int i = 0; i < P; i++) acc[i] = fmaf(wt, win[(j + i) % P], acc[i]);
        }
    }
}

__global__ void __launch_bounds__(32 * kGatherWX * kGatherWY, 1)
    lpaici_adjoint_gather_kernel(const __grid_constant__ GatherArgs a) {
    constexpr int P = kGatherP;
    extern __shared__ __align__(16) int smem[];
    __shared__ unsigned s_present;
    const int fsize = a.rows * a.pitch;
    int *s_blob = smem;
    float *s_c = reinterpret_cast<float *>(smem + a.blob_words);  // c_d on the halo'd tile
    float *s_f = s_c + fsize;                                     // the masked field of one scale
    uint8_t *s_s = reinterpret_cast<uint8_t *>(s_f + fsize);      // s*(d, .) on the halo'd tile
    const int x0 = blockIdx.x * kGatherTW, y0 = blockIdx.y * kGatherTH;
    const int gx0 = x0 - a.R, gy0 = y0 - a.R;

    stage_words(s_blob, a.blob, a.blob_words);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const int ty = (warp / kGatherWX) * 8 + (lane >> 2);
    const int tx = (warp % kGatherWX) * 4 * P + (lane & 3) * P;
    const int4 *s_runs = reinterpret_cast<const int4 *>(s_blob + a.run_word);
    const float *s_w = reinterpret_cast<const float *>(s_blob + a.weight_word);
    const float *lane_f = s_f + (ty + a.R) * a.pitch + tx + a.R;

    float acc[P];
#pragma unroll
    for (int i = 0; i < P; i++) acc[i] = 0.0f;

    for (int d = 0; d < a.D; d++) {
        __syncthreads();  // the previous direction's gathers are done with the shared fields
        if (threadIdx.x == 0) s_present = 0u;
        __syncthreads();
        unsigned present = 0;
        const uint8_t *plane = a.smap + static_cast<size_t>(d) * a.H * a.W;
        for (int r = warp; r < a.rows; r += nwarps) {  // one warp per row, lanes along it
            const int gy = gy0 + r;
            const bool row_ok = gy >= 0 && gy < a.H;
            for (int cc = lane; cc < a.pitch; cc += 32) {
                const int gx = gx0 + cc;
                float c = 0.0f;
                uint8_t s = 0xff;
                if (row_ok && gx >= 0 && gx < a.W) {
                    const size_t p = static_cast<size_t>(gy) * a.W + gx;
                    s = plane[p];
                    c = a.g[static_cast<size_t>(gy) * a.g_pitch + gx] * (a.rvar[d * a.S + s] / a.den[p]);
                    present |= 1u << s;
                }
                s_c[r * a.pitch + cc] = c;
                s_s[r * a.pitch + cc] = s;
            }
        }
        atomicOr(&s_present, present);
        __syncthreads();
        const unsigned mask = s_present;
        for (int s = 0; s < a.S; s++) {
            if (!(mask & (1u << s))) continue;  // block-uniform
            for (int i = threadIdx.x; i < fsize; i += blockDim.x) s_f[i] = (s_s[i] == s) ? s_c[i] : 0.0f;
            __syncthreads();
            const int k = d * a.S + s;
            for (int r = s_blob[k]; r < s_blob[k + 1]; r++) {
                const int4 run = s_runs[r];
                gather_run<P>(acc, lane_f + run.x * a.pitch + run.y, s_w + run.w, run.z);
            }
            __syncthreads();  // before the next scale's field overwrites s_f
        }
    }
    const int oy = y0 + ty;
    if (oy < a.H) {
        float *o = a.grad + static_cast<size_t>(oy) * a.grad_pitch + x0 + tx;
#pragma unroll
        for (int i = 0; i < P; i++)
            if (x0 + tx + i < a.W) o[i] = acc[i];
    }
}

}  // namespace

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
    if (ks->S > 32) return set_error(LPAICI_ERR_UNSUPPORTED, "lpaici_backward supports at most 32 scales");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const int *blob = nullptr, *adj = nullptr;
    int rc = device_blob(ks, &blob);
    if (rc == LPAICI_OK) rc = device_adj_blob(ks, &adj);
    if (rc != LPAICI_OK) return rc;

    // pass B's shared memory: mirrored kernels + c_d, masked field (floats) + s* (bytes) on the tile + halo
    GatherArgs ga{};
    ga.R = ks->radius;
    ga.pitch = field_pitch(kGatherTW + 2 * ga.R + kGatherP);
    ga.rows = kGatherTH + 2 * ga.R;
    ga.blob_words = static_cast<int>(ks->adj_blob.size());
    const size_t fsize = static_cast<size_t>(ga.pitch) * ga.rows;
    const size_t smem = sizeof(int) * ga.blob_words + 2 * sizeof(float) * fsize + fsize;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > static_cast<size_t>(max_optin))
        return set_error(LPAICI_ERR_UNSUPPORTED, "adjoint tile needs %zu B of shared memory, device allows %d", smem,
                         max_optin);

    // transient workspace: D selection planes (bytes) and den (floats)
    const size_t npx = static_cast<size_t>(width) * height;
    void *ws = nullptr;
    const size_t smap_bytes = (static_cast<size_t>(ks->D) * npx + 255) & ~size_t(255);
    cudaError_t e = cudaMallocAsync(&ws, smap_bytes + sizeof(float) * npx, stream);
    if (e != cudaSuccess) return cuda_error(e, "cudaMallocAsync(adjoint workspace)");
    uint8_t *smap = static_cast<uint8_t *>(ws);
    float *den = reinterpret_cast<float *>(static_cast<char *>(ws) + smap_bytes);

    // A. selection
    ImageArgs img{};
    img.in = d_noisy;
    img.out = nullptr;
    img.smap = smap;
    img.den = den;
    img.W = width;
    img.in_h = height;
    img.in_pitch = noisy_pitch;
    img.out_pitch = width;
    img.row_begin = 0;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    rc = launch_forward(ks, img, tab, default_config(ks), stream);

    // B. gather
    if (rc == LPAICI_OK) {
        ga.g = d_grad_out;
        ga.smap = smap;
        ga.den = den;
        ga.grad = d_grad_in;
        ga.g_pitch = gout_pitch;
        ga.grad_pitch = gin_pitch;
        ga.W = width;
        ga.H = height;
        ga.D = ks->D;
        ga.S = ks->S;
        ga.blob = adj;
        ga.run_word = ks->adj_run_word;
        ga.weight_word = ks->adj_weight_word;
        for (int k = 0; k < ks->D * ks->S; k++) ga.rvar[k] = 1.0f / tab.var[k];
        e = cudaFuncSetAttribute(lpaici_adjoint_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e == cudaSuccess) {
            const dim3 grid((width + kGatherTW - 1) / kGatherTW, (height + kGatherTH - 1) / kGatherTH);
            if (grid.y > 65535u) {
                rc = set_error(LPAICI_ERR_UNSUPPORTED, "image too tall: %d rows", height);
            } else {
                lpaici_adjoint_gather_kernel<<<grid, 32 * kGatherWX * kGatherWY, smem, stream>>>(ga);
                e = cudaGetLastError();
            }
        }
        if (rc == LPAICI_OK && e != cudaSuccess) rc = cuda_error(e, "adjoint gather launch");
    }
    cudaError_t ef = cudaFreeAsync(ws, stream);
    if (rc == LPAICI_OK && ef != cudaSuccess) rc = cuda_error(ef, "cudaFreeAsync(adjoint workspace)");
    return rc;
}

// The same two passes as lpaici_backward, over caller-provided storage (lpaici_backward_noalloc).
int lpaici::adjoint_passes(const lpaici_kernelset *ks, const int *blob, const int *adj_blob, uint8_t *smap,
                           float *den, const float *d_noisy, int noisy_pitch, const float *d_grad_out,
                           int gout_pitch, float *d_grad_in, int gin_pitch, int width, int height, float sigma,
                           float gamma, cudaStream_t stream) {
    GatherArgs ga{};
    ga.R = ks->radius;
    ga.pitch = field_pitch(kGatherTW + 2 * ga.R + kGatherP);
    ga.rows = kGatherTH + 2 * ga.R;
    ga.blob_words = static_cast<int>(ks->adj_blob.size());
    const size_t fsize = static_cast<size_t>(ga.pitch) * ga.rows;
    const size_t smem = sizeof(int) * ga.blob_words + 2 * sizeof(float) * fsize + fsize;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > static_cast<size_t>(max_optin))
        return set_error(LPAICI_ERR_UNSUPPORTED, "adjoint tile needs %zu B of shared memory, device allows %d", smem,
                         max_optin);
    const dim3 grid((width + kGatherTW - 1) / kGatherTW, (height + kGatherTH - 1) / kGatherTH);
    if (grid.y > 65535u) return set_error(LPAICI_ERR_UNSUPPORTED, "image too tall: %d rows", height);

    ImageArgs img{};
    img.in = d_noisy;
    img.out = nullptr;
    img.smap = smap;
    img.den = den;
    img.W = width;
    img.in_h = height;
    img.in_pitch = noisy_pitch;
    img.out_pitch = width;
    img.row_begin = 0;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    int rc = launch_forward(ks, img, tab, default_config(ks), stream);
    if (rc != LPAICI_OK) return rc;

    ga.g = d_grad_out;
    ga.smap = smap;
    ga.den = den;
    ga.grad = d_grad_in;
    ga.g_pitch = gout_pitch;
    ga.grad_pitch = gin_pitch;
    ga.W = width;
    ga.H = height;
    ga.D = ks->D;
    ga.S = ks->S;
    ga.blob = adj_blob;
    ga.run_word = ks->adj_run_word;
    ga.weight_word = ks->adj_weight_word;
    for (int k = 0; k < ks->D * ks->S; k++) ga.rvar[k] = 1.0f / tab.var[k];
    cudaError_t e = cudaFuncSetAttribute(lpaici_adjoint_gather_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_error(e, "adjoint gather attributes");
    lpaici_adjoint_gather_kernel<<<grid, 32 * kGatherWX * kGatherWY, smem, stream>>>(ga);
    e = cudaGetLastError();
    return e == cudaSuccess ? LPAICI_OK : cuda_error(e, "adjoint gather launch");
}
