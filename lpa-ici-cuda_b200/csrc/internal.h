// internal.h -- shared declarations of the LPA-ICI library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "lpaici.h"

namespace lpaici {

// Limits of this library.  The per-kernel variance and threshold tables travel as kernel
// parameters (2 * 4 B * kMaxKernels), so D*S is capped; the radius bounds the shared-memory halo.
constexpr int kMaxKernels = 256;
constexpr int kMaxRadius = 127;
// The sweeps keep each pixel's selected scale in 4 bits.
constexpr int kMaxScales = 16;

// One row run of a kernel, as the device reads it: the taps (dy, dx0 + j), j < len, whose weights
// are wdup[wofs + j] = {w_j, w_j}.  dy/dx0 are offsets from the output pixel
// (row - rows/2, col - cols/2); wofs is even, so two taps' duplicated weights are one 16-byte load.
struct Run {
    int dy, dx0, len, wofs;
};

// Device image of a kernel set, one contiguous block of 32-bit words:
//   [0, nk+1)               first run of kernel k (kernel k's runs are [begin[k], begin[k+1]))
//   [run_word, +4*n_runs)   Run records, 16-byte aligned
//   [weight_word, ...)      float2 {w, w} per tap, every run padded to an even number of taps
struct BlobLayout {
    int nk = 0, n_runs = 0, n_wdup = 0;
    int run_word = 0, weight_word = 0, total_words = 0;  // total padded to a multiple of 4
};

// Per-launch arguments shared by the forward and backward kernels (passed by value as a
// __grid_constant__ parameter; the tables are read with uniform indices from the constant bank).
struct ImageArgs {
    const float *in;  // input rows [0, in_h), width W, pitch in_pitch
    float *out;       // optional output rows [0, rows_out), pitch out_pitch
    uint8_t *smap;    // optional D x rows_out x W scale map
    float *rden;      // optional rows_out x W map of 1 / sum_d 1/v_d (pitch W; the adjoint's selection pass)
    int W, in_h, in_pitch, out_pitch;
    int row_begin;    // output row r is input row row_begin + r
    int rows_out;
    int step = 1;     // floats between neighbouring pixels of a row, in and out (channels of an interleaved image)
};

struct KernelTables {
    int D, S, R;
    float neg_zero;  // -0.0f, read at run time (see prod2 in tile_core.cuh)
    const int *blob;  // device blob (BlobLayout)
    int blob_words, run_word, weight_word;
    float var[kMaxKernels];
    float thr[kMaxKernels];
};

// Buffers of the images of a one-size batched plan (lpaici_forward_multi_kernel): image z's input,
// output, scale maps and 1/den (the last three may be null, as in ImageArgs).
constexpr int kMaxMultiImages = 64;
struct MultiImages {
    const float *in[kMaxMultiImages];
    float *out[kMaxMultiImages];
    uint8_t *smap[kMaxMultiImages];
    float *rden[kMaxMultiImages];
};

int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
// The checks every adjoint entry point makes before any copy or launch: sigma and gamma finite and
// positive (gamma only when the caller passes one), at most kMaxScales scales per direction (the
// selection sweep keeps each pixel's scale in 4 bits).  `who` names the entry point in the message.
int check_adjoint_params(const lpaici_kernelset *ks, float sigma, const float *gamma, const char *who);

}  // namespace lpaici

// The opaque kernel set of the C ABI.
struct lpaici_kernelset {
    int D = 0, S = 0;
    // the loader's dense output (load_LPA_kernels_standardized)
    std::vector<float> dense_w;
    std::vector<int> off, rows, cols;
    // the reference-layout run packing (build_sparse_kernels)
    std::vector<float> run_w;
    std::vector<int> run_row, run_col, run_len, k_first_run, k_num_runs, k_first_weight;
    // sum of squared weights per kernel, float, dense row-major order (compute_kernel_variances)
    std::vector<float> norm2;
    // nonzero taps per kernel (algorithmic work accounting)
    std::vector<int> nnz;
    int radius = 0;
    lpaici::BlobLayout layout;
    std::vector<int32_t> blob;  // host copy of the device blob
    // the adjoint gather's kernels, mirrored through their centre (taps (-dy, -dx)), in the forward
    // blob's layout (adj_layout): scale 0 as it is, every later scale as the difference from the scale
    // before it (kernelset.cpp, build_adjoint_blob)
    lpaici::BlobLayout adj_layout;
    std::vector<int32_t> adj_blob;
    // device copies, one per CUDA device, created on first use
    mutable std::mutex mu;
    mutable std::vector<int *> dev_blob;
    mutable std::vector<int *> dev_adj_blob;
    mutable std::vector<int> tuned_config;  // per device, -1 = not tuned
    // per device: ms one SM spends on one tile of each configuration, from lpaici_autotune (empty: not
    // tuned, or a configuration forced by lpaici_set_tile_config); and CTAs per SM of each (0: unknown)
    mutable std::vector<std::vector<float>> tuned_tile_ms;
    mutable std::vector<std::vector<int>> blocks_per_sm;
};

namespace lpaici {

// Device blob of ks on the current device (uploaded on first use).  Returns an LPAICI_* code.
int device_blob(const lpaici_kernelset *ks, const int **out);
// The adjoint's flipped-kernel blob on the current device (uploaded on first use).
int device_adj_blob(const lpaici_kernelset *ks, const int **out);

// Fills var/thr exactly as the reference: var = (sigma*sigma)*norm2, thr = gamma*sqrt(var).
void fill_tables(const lpaici_kernelset *ks, const float *var_or_null, float sigma, float gamma, KernelTables *t);

// Forward / backward launchers (forward.cu, backward.cu).
// fused: each tap one fused multiply-add instead of a rounded product and a rounded sum (faster, not
// bit-exact with the reference: lpaici_forward_ffma).
int launch_forward(const lpaici_kernelset *ks, const ImageArgs &img, const KernelTables &tab, int config,
                   cudaStream_t stream, bool fused = false);
// n images of img's size, pitches and tables (tab) in one launch, their buffers in mi.
int launch_forward_multi(const ImageArgs &img, const KernelTables &tab, const MultiImages &mi, int n, int config,
                         cudaStream_t stream);
// Bytes of shared memory tile configuration `config` needs for a kernel set.
size_t config_smem(int config, int blob_words, int nk, int R);
// The autotuned configuration of ks on the current device, else the first one that fits.
int default_config(const lpaici_kernelset *ks);
// The configuration expected to be fastest for one launch over width x rows pixels: per-tile time
// (tuned, else a B200 table) times the waves of CTAs the image needs.  A forced configuration wins.
int config_for(const lpaici_kernelset *ks, int width, int rows);
// The same for one launch over n images (a batched plan's tile queue): the images' tiles add up.
int config_for_images(const lpaici_kernelset *ks, const int *widths, const int *rows, int n);
// CTAs of the forward kernel of `config` that fit on one SM with `smem` bytes of shared memory.
int config_blocks_per_sm(int config, size_t smem);
// Tile width and height of a configuration.
void config_tile(int config, int *tile_w, int *tile_h);
// One image of a batch plan (batched.cu): out may be null (no estimate), smap and rden optional.
struct BatchSpec {
    const float *noisy;
    float *out;
    uint8_t *smap;
    float *rden;
    int width, height, noisy_pitch, out_pitch;
    float sigma, gamma;
};
int batch_plan_create(const lpaici_kernelset *ks, const BatchSpec *specs, int n, int config, bool use_graph,
                      cudaStream_t stream, lpaici_batch **out);
int batch_plan_enqueue(lpaici_batch *b, cudaStream_t stream);  // queue reset + persistent launch
void batch_plan_free(lpaici_batch *b);

// The adjoint's two passes over storage the caller provides: device copies of ks->blob and ks->adj_blob,
// D*width*height selection bytes and width*height floats of 1/den.  Allocates nothing.
int adjoint_passes(const lpaici_kernelset *ks, const int *blob, const int *adj_blob, uint8_t *smap, float *rden,
                   const float *d_noisy, int noisy_pitch, const float *d_grad_out, int gout_pitch, float *d_grad_in,
                   int gin_pitch, int width, int height, float sigma, float gamma, cudaStream_t stream);

}  // namespace lpaici
