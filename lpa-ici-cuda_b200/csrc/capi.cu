// capi.cu -- C ABI entry points for the forward path, the reference-shaped host engine and the
// tile-configuration table.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "configs.h"
#include "internal.h"

using namespace lpaici;

namespace lpaici {

int default_config(const lpaici_kernelset *ks) {
    int dev = 0, max_optin = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) {
        std::lock_guard<std::mutex> lock(ks->mu);
        if (dev < static_cast<int>(ks->tuned_config.size()) && ks->tuned_config[dev] >= 0)
            return ks->tuned_config[dev];
    }
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    static const int order[] = LPAICI_TILE_PREFERENCE;
    static_assert(sizeof(order) / sizeof(order[0]) == LPAICI_NUM_TILE_CONFIGS, "one preference per configuration");
    for (const int c : order)
        if (config_smem(c, ks->layout.total_words, ks->D * ks->S, ks->radius) <= static_cast<size_t>(max_optin))
            return c;
    return LPAICI_DEFAULT_TILE_CONFIG;  // nothing fits: the launch reports LPAICI_ERR_UNSUPPORTED
}

// ms one B200 SM (1,965 MHz) spends on one tile of each configuration, measured on the 4096^2
// benchmark image with the 16x7 symmetric kernels (launch time / waves): the estimate for kernel sets
// that were not tuned.
static const float kTileMs[LPAICI_NUM_TILE_CONFIGS] = {0.349f, 0.350f, 0.357f, 0.426f, 0.427f, 0.442f,
                                                0.261f, 0.412f, 0.412f, 0.485f, 0.479f};

// CTAs per SM of configuration c for ks on device dev (cached; 0 when it does not fit).
static int cached_bps(const lpaici_kernelset *ks, int dev, int c, int max_optin) {
    {
        std::lock_guard<std::mutex> lock(ks->mu);
        if (dev < static_cast<int>(ks->blocks_per_sm.size()) && !ks->blocks_per_sm[dev].empty() &&
            ks->blocks_per_sm[dev][c] >= 0)
            return ks->blocks_per_sm[dev][c];
    }
    const size_t smem = config_smem(c, ks->layout.total_words, ks->D * ks->S, ks->radius);
    const int n = smem <= static_cast<size_t>(max_optin) ? config_blocks_per_sm(c, smem) : 0;
    std::lock_guard<std::mutex> lock(ks->mu);
    if (static_cast<int>(ks->blocks_per_sm.size()) <= dev) ks->blocks_per_sm.resize(dev + 1);
    if (ks->blocks_per_sm[dev].empty()) ks->blocks_per_sm[dev].assign(LPAICI_NUM_TILE_CONFIGS, -1);
    ks->blocks_per_sm[dev][c] = n;
    return n;
}

static long tiles_of(int c, int width, int rows) {
    int tw = 1, th = 1;
    config_tile(c, &tw, &th);
    return static_cast<long>((width + tw - 1) / tw) * ((rows + th - 1) / th);
}

int config_for_images(const lpaici_kernelset *ks, const int *widths, const int *rows, int n) {
    int dev = 0, sms = 0, max_optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return default_config(ks);
    std::vector<float> tuned;
    {
        std::lock_guard<std::mutex> lock(ks->mu);
        const bool have = dev < static_cast<int>(ks->tuned_config.size()) && ks->tuned_config[dev] >= 0;
        const bool timed = dev < static_cast<int>(ks->tuned_tile_ms.size()) && !ks->tuned_tile_ms[dev].empty();
        if (have && !timed) return ks->tuned_config[dev];  // forced by lpaici_set_tile_config
        if (timed) tuned = ks->tuned_tile_ms[dev];
    }
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    int best = -1;
    double best_ms = 0.0;
    for (int c = 0; c < LPAICI_NUM_TILE_CONFIGS; c++) {
        const int bps = cached_bps(ks, dev, c, max_optin);
        const float tile_ms = tuned.empty() ? kTileMs[c] : tuned[c];
        if (bps <= 0 || !(tile_ms > 0.0f)) continue;
        long tiles = 0;
        for (int i = 0; i < n; i++) tiles += tiles_of(c, widths[i], rows[i]);
        const long slots = static_cast<long>(sms) * bps;
        const double est = tile_ms * bps * static_cast<double>((tiles + slots - 1) / slots);
        if (best < 0 || est < best_ms) {
            best = c;
            best_ms = est;
        }
    }
    return best >= 0 ? best : default_config(ks);
}

int config_for(const lpaici_kernelset *ks, int width, int rows) { return config_for_images(ks, &width, &rows, 1); }

static int check_params(float sigma_or_one, float gamma) {
    if (!(sigma_or_one > 0.0f) || !std::isfinite(sigma_or_one))
        return set_error(LPAICI_ERR_INVALID_ARG, "sigma needs a positive number, got %g", sigma_or_one);
    if (!(gamma > 0.0f) || !std::isfinite(gamma))
        return set_error(LPAICI_ERR_INVALID_ARG, "gamma needs a positive number, got %g", gamma);
    return LPAICI_OK;
}

// Shared body of the forward entry points.
static int forward_common(const lpaici_kernelset *ks, const float *d_in, int in_pitch, int width, int in_height,
                          int row_begin, int row_count, float *d_out, int out_pitch, const float *host_var,
                          float sigma, float gamma, uint8_t *d_smap, cudaStream_t stream, int step = 1,
                          int config = -1, bool fused = false) {
    if (!ks || !d_in || !d_out) return set_error(LPAICI_ERR_INVALID_ARG, "forward: null kernel set or image pointer");
    if (width <= 0 || in_height <= 0 || row_count <= 0)
        return set_error(LPAICI_ERR_INVALID_ARG, "forward: non-positive size %d x %d", width, row_count);
    const long row_floats = static_cast<long>(width - 1) * step + 1;
    if (in_pitch < row_floats || out_pitch < row_floats)
        return set_error(LPAICI_ERR_INVALID_ARG, "forward: pitch smaller than width");
    if (row_begin < 0 || row_begin + row_count > in_height)
        return set_error(LPAICI_ERR_INVALID_ARG, "forward: output rows [%d, %d) outside the %d input rows", row_begin,
                         row_begin + row_count, in_height);
    int rc = check_params(host_var ? 1.0f : sigma, gamma);
    if (rc != LPAICI_OK) return rc;
    if (host_var)
        for (int k = 0; k < ks->D * ks->S; k++)
            if (!(host_var[k] >= 0.0f))
                return set_error(LPAICI_ERR_INVALID_ARG, "forward: variance %d is %g", k, host_var[k]);
    const int *blob = nullptr;
    rc = device_blob(ks, &blob);
    if (rc != LPAICI_OK) return rc;
    ImageArgs img{};
    img.in = d_in;
    img.out = d_out;
    img.smap = d_smap;
    img.W = width;
    img.in_h = in_height;
    img.in_pitch = in_pitch;
    img.out_pitch = out_pitch;
    img.row_begin = row_begin;
    img.rows_out = row_count;
    img.step = step;
    KernelTables tab;
    fill_tables(ks, host_var, sigma, gamma, &tab);
    tab.blob = blob;
    return launch_forward(ks, img, tab, config >= 0 ? config : config_for(ks, width, row_count), stream, fused);
}

// Every channel of an interleaved image (pixel (x, y), channel c at row y, float x * channels + c) as
// its own image, in place: one launch per channel with element stride `channels`.
static int forward_channels(const lpaici_kernelset *ks, const float *d_in, int in_pitch, float *d_out, int out_pitch,
                            int width, int height, int channels, const float *host_var, float sigma, float gamma,
                            cudaStream_t stream) {
    if (channels <= 0 || channels > 64)
        return set_error(LPAICI_ERR_INVALID_ARG, "channels must be 1 .. 64, got %d", channels);
    for (int c = 0; c < channels; c++) {
        const int rc = forward_common(ks, d_in ? d_in + c : nullptr, in_pitch, width, height, 0, height,
                                      d_out ? d_out + c : nullptr, out_pitch, host_var, sigma, gamma, nullptr, stream,
                                      channels);
        if (rc != LPAICI_OK) return rc;
    }
    return LPAICI_OK;
}

}  // namespace lpaici

extern "C" {

int lpaici_forward(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                   int out_pitch, int width, int height, float sigma, float gamma, uint8_t *d_scale_map,
                   lpaici_stream_t stream) {
    return forward_common(ks, d_noisy, noisy_pitch, width, height, 0, height, d_denoised, out_pitch, nullptr, sigma,
                          gamma, d_scale_map, reinterpret_cast<cudaStream_t>(stream));
}

int lpaici_forward_ffma(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                        int out_pitch, int width, int height, float sigma, float gamma, uint8_t *d_scale_map,
                        lpaici_stream_t stream) {
    return forward_common(ks, d_noisy, noisy_pitch, width, height, 0, height, d_denoised, out_pitch, nullptr, sigma,
                          gamma, d_scale_map, reinterpret_cast<cudaStream_t>(stream), 1, -1, true);
}

int lpaici_forward_var(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                       int out_pitch, int width, int height, const float *host_var, float gamma,
                       uint8_t *d_scale_map, lpaici_stream_t stream) {
    if (!host_var) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_forward_var: null variances");
    return forward_common(ks, d_noisy, noisy_pitch, width, height, 0, height, d_denoised, out_pitch, host_var, 1.0f,
                          gamma, d_scale_map, reinterpret_cast<cudaStream_t>(stream));
}

int lpaici_forward_rows(const lpaici_kernelset *ks, const float *d_in, int in_pitch, int width, int in_height,
                        int row_begin, int row_count, float *d_out, int out_pitch, float sigma, float gamma,
                        uint8_t *d_scale_map, lpaici_stream_t stream) {
    return forward_common(ks, d_in, in_pitch, width, in_height, row_begin, row_count, d_out, out_pitch, nullptr, sigma,
                          gamma, d_scale_map, reinterpret_cast<cudaStream_t>(stream));
}

int lpaici_forward_channels(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                            int out_pitch, int width, int height, int channels, float sigma, float gamma,
                            lpaici_stream_t stream) {
    return forward_channels(ks, d_noisy, noisy_pitch, d_denoised, out_pitch, width, height, channels, nullptr, sigma,
                            gamma, reinterpret_cast<cudaStream_t>(stream));
}

int lpaici_num_tile_configs(void) { return LPAICI_NUM_TILE_CONFIGS; }

int lpaici_tile_config_desc(int index, int *tile_w, int *tile_h, int *threads, int *pixels_per_thread) {
#define LPAICI_DESC_CASE(idx, WX, WY, Q)                  \
    case idx:                                             \
        if (tile_w) *tile_w = (WX) * 4 * (Q);             \
        if (tile_h) *tile_h = (WY) * 16;                  \
        if (threads) *threads = 32 * (WX) * (WY);         \
        if (pixels_per_thread) *pixels_per_thread = 2 * (Q); \
        return LPAICI_OK;
    switch (index) {
        LPAICI_TILE_CONFIGS(LPAICI_DESC_CASE)
        default: return set_error(LPAICI_ERR_INVALID_ARG, "tile config %d out of range", index);
    }
#undef LPAICI_DESC_CASE
}

// ---- host-pointer engines ---------------------------------------------------------------------

namespace {
// Device buffers of lpaici_denoise_host, per thread and device.
// Device buffers and the copy/compute pipeline of lpaici_denoise_host, per host thread and device.
constexpr int kMaxBands = 64;
struct HostBuffers {
    int dev = -1;
    float *in = nullptr, *out = nullptr;
    size_t cap = 0;
    cudaStream_t s_in = nullptr, s_out = nullptr, s_comp[2] = {nullptr, nullptr};
    cudaEvent_t ev_start = nullptr, ev_done = nullptr, ev_in[kMaxBands] = {}, ev_comp[kMaxBands] = {};
    ~HostBuffers() { release(); }
    void release() {
        if (dev >= 0) {
            int cur = -1;
            cudaGetDevice(&cur);
            cudaSetDevice(dev);
            cudaFree(in);
            cudaFree(out);
            for (cudaStream_t st : {s_in, s_out, s_comp[0], s_comp[1]})
                if (st) cudaStreamDestroy(st);
            for (cudaEvent_t ev : {ev_start, ev_done})
                if (ev) cudaEventDestroy(ev);
            for (int i = 0; i < kMaxBands; i++) {
                if (ev_in[i]) cudaEventDestroy(ev_in[i]);
                if (ev_comp[i]) cudaEventDestroy(ev_comp[i]);
                ev_in[i] = ev_comp[i] = nullptr;
            }
            if (cur >= 0) cudaSetDevice(cur);
        }
        in = out = nullptr;
        s_in = s_out = s_comp[0] = s_comp[1] = nullptr;
        ev_start = ev_done = nullptr;
        cap = 0;
        dev = -1;
    }
    cudaError_t make_pipeline() {
        cudaError_t e = cudaSuccess;
        for (cudaStream_t *st : {&s_in, &s_out, &s_comp[0], &s_comp[1]})
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
        for (cudaEvent_t *ev : {&ev_start, &ev_done})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        for (int i = 0; i < kMaxBands && e == cudaSuccess; i++) {
            e = cudaEventCreateWithFlags(&ev_in[i], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_comp[i], cudaEventDisableTiming);
        }
        return e;
    }
};
thread_local HostBuffers t_bufs;
}  // namespace

int lpaici_denoise_host(const lpaici_kernelset *ks, const float *host_noisy, float *host_denoised, int width,
                        int height, float sigma, float gamma, lpaici_stream_t stream_) {
    if (!ks || !host_noisy || !host_denoised || width <= 0 || height <= 0)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_denoise_host: bad argument");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    int rc = check_params(sigma, gamma);
    if (rc != LPAICI_OK) return rc;
    const size_t n = static_cast<size_t>(width) * height;
    if (t_bufs.dev != dev || t_bufs.cap < n) {
        t_bufs.release();
        t_bufs.dev = dev;
        e = cudaMalloc(&t_bufs.in, n * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&t_bufs.out, n * sizeof(float));
        if (e == cudaSuccess) e = t_bufs.make_pipeline();
        if (e != cudaSuccess) {
            t_bufs.release();
            return cuda_error(e, "host-pointer buffers");
        }
        t_bufs.cap = n;
    }
    // Row bands, pipelined: the upload of the rows band b needs (its rows + R below) on s_in, its
    // forward on one of two compute streams (the next band's CTAs fill the SMs while this band's last
    // wave drains), its download on s_out.  With pinned host buffers the copies overlap the kernels.
    // one configuration for all bands, chosen for the whole image: the bands' launches overlap on two
    // streams, so the GPU sees one stream of tiles, not separate short launches
    const int config = config_for(ks, width, height);
    int tile_h = 64;
    lpaici_tile_config_desc(config, nullptr, &tile_h, nullptr, nullptr);
    const int R = ks->radius;
    // band i covers rows [edge[i], edge[i + 1]): the first is one tile row high and the last one or two,
    // so the upload before the first forward and the download after the last one are short; the
    // bands between are about an eighth of the image
    int edge[kMaxBands + 1];
    int nb = 0;
    if (height <= 3 * tile_h) {
        edge[0] = 0;
        edge[1] = height;
        nb = 1;
    } else {
        const int last = tile_h + (height - 2 * tile_h) % tile_h;  // the middle bands stay whole tile rows
        const int mid = height - tile_h - last;
        int band = ((height + 7) / 8 + tile_h - 1) / tile_h * tile_h;
        while (2 + (mid + band - 1) / band > kMaxBands) band += tile_h;
        edge[0] = 0;
        edge[1] = tile_h;
        nb = 1;
        for (int r = tile_h; r < tile_h + mid; r += band) edge[++nb] = std::min(tile_h + mid, r + band);
        edge[++nb] = height;
    }
    HostBuffers &b = t_bufs;
    e = cudaEventRecord(b.ev_start, stream);
    for (cudaStream_t st : {b.s_in, b.s_out, b.s_comp[0], b.s_comp[1]})
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b.ev_start, 0);
    if (e != cudaSuccess) return cuda_error(e, "lpaici_denoise_host: stream order");
    int copied = 0;  // input rows [0, copied) uploaded
    for (int i = 0; i < nb && rc == LPAICI_OK; i++) {
        const int r0 = edge[i], r1 = edge[i + 1], need = std::min(height, r1 + R);
        if (need > copied) {
            e = cudaMemcpyAsync(b.in + static_cast<size_t>(copied) * width, host_noisy + static_cast<size_t>(copied) * width,
                                sizeof(float) * width * static_cast<size_t>(need - copied), cudaMemcpyHostToDevice, b.s_in);
            copied = need;
        }
        if (e == cudaSuccess) e = cudaEventRecord(b.ev_in[i], b.s_in);
        cudaStream_t sc = b.s_comp[i & 1];
        if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, b.ev_in[i], 0);
        if (e != cudaSuccess) {
            rc = cuda_error(e, "lpaici_denoise_host: upload");
            break;
        }
        rc = forward_common(ks, b.in, width, width, height, r0, r1 - r0, b.out + static_cast<size_t>(r0) * width, width,
                            nullptr, sigma, gamma, nullptr, sc, 1, config);
        if (rc != LPAICI_OK) break;
        e = cudaEventRecord(b.ev_comp[i], sc);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b.s_out, b.ev_comp[i], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host_denoised + static_cast<size_t>(r0) * width, b.out + static_cast<size_t>(r0) * width,
                                sizeof(float) * width * static_cast<size_t>(r1 - r0), cudaMemcpyDeviceToHost, b.s_out);
        if (e != cudaSuccess) rc = cuda_error(e, "lpaici_denoise_host: download");
    }
    // every band's download waited for its forward, every forward for its upload: s_out covers all
    e = cudaEventRecord(b.ev_done, b.s_out);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, b.ev_done, 0);
    const cudaError_t es = cudaStreamSynchronize(b.s_out);
    if (rc != LPAICI_OK) return rc;
    if (e != cudaSuccess) return cuda_error(e, "lpaici_denoise_host: join");
    if (es != cudaSuccess) return cuda_error(es, "cudaStreamSynchronize");
    return LPAICI_OK;
}

int lpaici_release_host_buffers(void) {
    t_bufs.release();
    return LPAICI_OK;
}

int lpaici_anisotropic_gpu_fused(float *host_img_noisy, float *host_img_denoised, int width, int height, int channels,
                                 float *host_global_weights_buffer, int num_dirs, int num_scales,
                                 float *host_kernel_weights, int host_kernel_weights_size, int *host_offsets,
                                 int *host_rows, int *host_cols, float *host_kernel_variances, float ici_gamma,
                                 double *seconds) {
    (void)host_global_weights_buffer;
    if (channels <= 0 || channels > 64)
        return set_error(LPAICI_ERR_INVALID_ARG, "channels must be 1 .. 64, got %d", channels);
    if (!host_img_noisy || !host_img_denoised || !host_kernel_weights || !host_offsets || !host_rows || !host_cols ||
        !host_kernel_variances || width <= 0 || height <= 0)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_anisotropic_gpu_fused: bad argument");
    const long nk = static_cast<long>(num_dirs) * num_scales;
    for (long k = 0; k < nk; k++)
        if (host_offsets[k] < 0 || static_cast<long>(host_offsets[k]) + static_cast<long>(host_rows[k]) * host_cols[k] >
                                       host_kernel_weights_size)
            return set_error(LPAICI_ERR_KERNEL_FORMAT, "kernel %ld lies outside the %d weights", k,
                             host_kernel_weights_size);
    lpaici_kernelset *ks = nullptr;
    int rc = lpaici_kernelset_create(host_kernel_weights, host_offsets, host_rows, host_cols, num_dirs, num_scales, &ks);
    if (rc != LPAICI_OK) return rc;
    const size_t n = static_cast<size_t>(width) * height * channels;
    float *d_in = nullptr, *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_in, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(d_in, host_img_noisy, n * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        rc = cuda_error(e, "lpaici_anisotropic_gpu_fused setup");
    } else {
        cudaDeviceSynchronize();
        const auto t0 = std::chrono::steady_clock::now();  // the reference's window starts here (:1216)
        rc = forward_channels(ks, d_in, width * channels, d_out, width * channels, width, height, channels,
                              host_kernel_variances, 1.0f, ici_gamma, nullptr);
        if (rc == LPAICI_OK) {
            e = cudaMemcpy(host_img_denoised, d_out, n * sizeof(float), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = cuda_error(e, "cudaMemcpy(D2H)");
        }
        const auto t1 = std::chrono::steady_clock::now();  // ... and ends after the copy back (:1240)
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    }
    cudaFree(d_in);
    cudaFree(d_out);
    lpaici_kernelset_destroy(ks);
    return rc;
}

}  // extern "C"

// ---- autotuner ----------------------------------------------------------------------------------

namespace {

// Built-in tuning image: a smooth ramp, a stripe texture and blocks, plus hash noise of 0.08.
__global__ void synth_tuning_image(float *img, int W, int H, int pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    unsigned h = static_cast<unsigned>(x) * 0x9E3779B1u ^ static_cast<unsigned>(y) * 0x85EBCA77u;
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    const float u = (h & 0xFFFFFF) * (1.0f / 16777216.0f) - 0.5f;
    const float ramp = 0.3f * x / W + 0.2f * y / H;
    const float stripes = 0.2f * sinf(0.7f * x + 0.4f * y);
    const float block = (((x >> 7) ^ (y >> 7)) & 1) ? 0.3f : 0.0f;
    img[static_cast<size_t>(y) * pitch + x] = ramp + stripes + block + 0.28f * u;
}

}  // namespace

extern "C" int lpaici_autotune(lpaici_kernelset *ks, const float *d_sample, int width, int height, int pitch,
                               float sigma, float gamma, int reps, int *best_config, float *ms_out,
                               lpaici_stream_t stream_) {
    if (!ks || width <= 0 || height <= 0 || (d_sample && pitch < width) || reps <= 0)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_autotune: bad argument");
    int rc = check_params(sigma, gamma);
    if (rc != LPAICI_OK) return rc;
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    const size_t n = static_cast<size_t>(width) * height;
    float *in = nullptr, *out = nullptr;
    cudaError_t e = cudaSuccess;
    if (!d_sample) {
        e = cudaMalloc(&in, n * sizeof(float));
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc(autotune)");
        synth_tuning_image<<<dim3((width + 255) / 256, height), 256, 0, stream>>>(in, width, height, width);
        pitch = width;
    }
    e = cudaMalloc(&out, n * sizeof(float));
    if (e != cudaSuccess) {
        cudaFree(in);
        return cuda_error(e, "cudaMalloc(autotune)");
    }
    const float *src = d_sample ? d_sample : in;
    const int *blob = nullptr;
    rc = device_blob(ks, &blob);
    ImageArgs img{};
    img.in = src;
    img.out = out;
    img.W = width;
    img.in_h = height;
    img.in_pitch = pitch;
    img.out_pitch = width;
    img.rows_out = height;
    KernelTables tab;
    fill_tables(ks, nullptr, sigma, gamma, &tab);
    tab.blob = blob;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 0.0f;
    int best = -1;
    std::vector<float> config_ms(LPAICI_NUM_TILE_CONFIGS, -1.0f);
    for (int c = 0; rc == LPAICI_OK && c < LPAICI_NUM_TILE_CONFIGS; c++) {
        int crc = launch_forward(ks, img, tab, c, stream);  // warm-up
        if (crc != LPAICI_OK) {
            if (ms_out) ms_out[c] = -1.0f;
            if (crc == LPAICI_ERR_UNSUPPORTED) continue;  // this tile does not fit for this kernel set
            rc = crc;
            break;
        }
        cudaEventRecord(e0, stream);
        for (int r = 0; r < reps && crc == LPAICI_OK; r++) crc = launch_forward(ks, img, tab, c, stream);
        cudaEventRecord(e1, stream);
        e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            rc = cuda_error(e, "autotune");
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= reps;
        if (ms_out) ms_out[c] = ms;
        config_ms[c] = ms;
        if (best < 0 || ms < best_ms) {
            best = c;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(in);
    cudaFree(out);
    if (rc != LPAICI_OK) return rc;
    if (best < 0) return set_error(LPAICI_ERR_UNSUPPORTED, "no tile configuration fits this kernel set");
    if (best_config) *best_config = best;
    rc = lpaici_set_tile_config(ks, best);
    if (rc != LPAICI_OK) return rc;
    // per-tile times, for picking the configuration of other image sizes (config_for)
    int dev = 0, sms = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    std::vector<float> tile_ms(LPAICI_NUM_TILE_CONFIGS, -1.0f);
    for (int c = 0; c < LPAICI_NUM_TILE_CONFIGS; c++) {
        const int bps = cached_bps(ks, dev, c, max_optin);
        if (!(config_ms[c] > 0.0f) || bps <= 0) continue;
        const long slots = static_cast<long>(sms) * bps;
        tile_ms[c] = config_ms[c] / (bps * static_cast<float>((tiles_of(c, width, height) + slots - 1) / slots));
    }
    std::lock_guard<std::mutex> lock(ks->mu);
    if (static_cast<int>(ks->tuned_tile_ms.size()) <= dev) ks->tuned_tile_ms.resize(dev + 1);
    ks->tuned_tile_ms[dev] = tile_ms;
    return LPAICI_OK;
}

extern "C" int lpaici_set_tile_config(lpaici_kernelset *ks, int config) {
    if (!ks || config < -1 || config >= LPAICI_NUM_TILE_CONFIGS)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_set_tile_config: bad argument");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(ks->mu);
    if (static_cast<int>(ks->tuned_config.size()) <= dev) {
        ks->dev_blob.resize(dev + 1, nullptr);
        ks->tuned_config.resize(dev + 1, -1);
    }
    ks->tuned_config[dev] = config;
    if (dev < static_cast<int>(ks->tuned_tile_ms.size())) ks->tuned_tile_ms[dev].clear();  // forced
    return LPAICI_OK;
}
