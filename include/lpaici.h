/*
 * lpaici.h -- C ABI of the B200 LPA-ICI denoiser (anisotropic Local Polynomial Approximation with
 * Intersection of Confidence Intervals).
 *
 * Plain C: no C++ or torch types cross this boundary; pointers, sizes and a status code.
 * Every entry point returns LPAICI_OK (0) or a nonzero LPAICI_ERR_* code and never exits the
 * process; lpaici_last_error() gives a message for the calling thread's last failure.
 *
 * Device entry points take device pointers owned by the caller and run on the CUDA device that is
 * current on the calling thread, asynchronously on the given stream (NULL = legacy default stream).
 * A kernel set is immutable once created, so concurrent calls on different streams or threads are
 * safe.  The reference these entry points replace is titocapovilla/lpa-ici-cuda; each declaration
 * cites the function (file:line) whose behaviour it reproduces.
 *
 * Arithmetic: every result is bit-identical to the reference's CPU path
 * (src/v1_0_lpa_ici_2D_fused.cpp:803-930) for finite inputs: the taps of each kernel are summed in
 * row-major order with separately rounded multiply and add, bounds, threshold (gamma*sqrt(var)),
 * reciprocal weights and the final division all round exactly as the reference's do.
 */
#ifndef LPAICI_H
#define LPAICI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LPAICI_VERSION_MAJOR 1
#define LPAICI_VERSION_MINOR 0

/* ---- status codes ------------------------------------------------------------------------- */
#define LPAICI_OK 0
#define LPAICI_ERR_INVALID_ARG 1    /* null pointer, size <= 0, sigma/gamma not > 0, channels outside 1..64 ... */
#define LPAICI_ERR_FILE 2           /* a file cannot be opened / read / written */
#define LPAICI_ERR_KERNEL_FORMAT 3  /* malformed kernel file or kernel arrays */
#define LPAICI_ERR_UNSUPPORTED 4    /* valid input beyond this build's limits (e.g. kernel radius) */
#define LPAICI_ERR_CUDA 5           /* a CUDA runtime call failed */
#define LPAICI_ERR_NO_MEMORY 6      /* host or device allocation failed */

/* cudaStream_t without the CUDA headers (cudaStream_t is a struct CUstream_st pointer). */
typedef struct CUstream_st *lpaici_stream_t;

/* Message of the calling thread's last failure ("" if none).  Valid until the next call. */
const char *lpaici_last_error(void);
/* Constant name of a status code. */
const char *lpaici_status_string(int status);

/* ---- kernel sets ---------------------------------------------------------------------------- */
typedef struct lpaici_kernelset lpaici_kernelset;

typedef struct {
    int num_dirs;     /* D */
    int num_scales;   /* S */
    int dense_size;   /* sum over kernels of rows*cols (the reference's host_kernel_weights_size) */
    int n_taps;       /* weights kept by the run-length packer (nonzeros + interior zeros of runs) */
    int n_runs;       /* row runs over all kernels */
    int radius;       /* largest |tap offset| from the kernel centre, rows or columns */
    int blob_bytes;   /* device copy of the forward's packed kernels (one per device, made on first use) */
    int adjoint_blob_bytes; /* device copy of the adjoint's mirrored kernels (one per device) */
} lpaici_kernelset_info_t;

/* Reads a kernel file: "D S", then D*S blocks "rows cols w[rows*cols]" in row-major order, and
 * centre-crops every direction to direction 0's size at the same scale.  Packs every kernel row
 * into one run from its first to its last nonzero, in global memory (no size cap).
 * Replaces load_LPA_kernels_standardized (src/v1_0_lpa_ici_2D_fused.cpp:466-551) +
 * build_sparse_kernels (src/v4_1_lpa_ici_2D_sparse_shared.cu:826-877) + the constant-memory
 * upload and its capacity checks (src/v4_1_lpa_ici_2D_sparse_shared.cu:1175-1214).
 * Errors: LPAICI_ERR_FILE (cannot open), LPAICI_ERR_KERNEL_FORMAT (bad header, size or weights,
 * or a kernel smaller than direction 0's at its scale), LPAICI_ERR_UNSUPPORTED (radius > 127; the
 * launches refuse radii whose halo'd tile does not fit in shared memory, about 48-60). */
int lpaici_kernelset_load(const char *path, lpaici_kernelset **out);

/* Builds a kernel set from the loader's dense arrays (weights, offsets, rows, cols: D*S kernels,
 * kernel k = d*S + s at weights[offsets[k]], rows[k] x cols[k] row-major), the form the
 * reference's engine takes (src/v4_1_lpa_ici_2D_sparse_shared.cu:1122-1132). */
int lpaici_kernelset_create(const float *weights, const int *offsets, const int *rows, const int *cols,
                            int num_dirs, int num_scales, lpaici_kernelset **out);

/* Writes the kernel set as a binary tap-list file: the kernel sizes and the run-length packing (the
 * packer's runs and weights, little-endian, FNV-1a checked).  lpaici_kernelset_load reads such a file
 * as well as the text format (it tells them apart by the file's first 8 bytes, "LPAICIT1"), and the
 * command line's -k accepts it: the loader skips the text parse and rebuilds the same kernel set
 * (dense values outside the runs come back as +0).  No counterpart in the reference. */
int lpaici_kernelset_save(const lpaici_kernelset *ks, const char *path);

/* Kernel generation.  The reference ships its kernel files precomputed by a MATLAB LASIP script that is
 * not in its tree (readme.md "Kernel files"); this generates directional LPA kernels of the same form
 * from their definition: D directions (direction d points at angle 2*pi*d/D, counter-clockwise from +x,
 * image rows down), one kernel per scale h = scales[s] on a (2h-1) x (2h-1) grid centred on the pixel.
 * With u the distance along the direction and v across it, the support is
 *   LPAICI_SHAPE_SECTOR:   the origin and every pixel with u < h - 1/2 whose angle from the direction
 *                          is at most pi/D (a wedge, the directions tiling the plane);
 *   LPAICI_SHAPE_QUADRANT: 0 <= u <= h - 1 and -(h - 1) <= v <= 0 (an h x h square on one side);
 * and the weights are the local polynomial approximation of order `order` in u (0 .. 4; lowered to the
 * number of distinct u values less one) with a uniform window, evaluated at the pixel: the least-squares
 * fit of sum_q b_q u^q to the support, whose weights sum to 1.  Order 0 sectors reproduce
 * kernels/lpa_kernels_m_1_0_d_16_h12_1_2_4_8_16_24_32_symmetric.txt (the default set), order 0 and 1
 * quadrants the d_4_square sets, once written as text and read back (lpaici_kernelset_write_text prints 6
 * decimals, as those files do): bit for bit, up to the sign of weights that are zero in exact arithmetic.  The Gaussian-window sets are not
 * of this form.  No counterpart in the reference's code. */
#define LPAICI_SHAPE_SECTOR 0
#define LPAICI_SHAPE_QUADRANT 1
int lpaici_kernelset_generate(int num_dirs, int num_scales, const int *scales, int order, int shape,
                              lpaici_kernelset **out);

/* Writes the dense kernels in the reference's text format (readme.md:95-103): "D S", then per kernel
 * "rows cols" and its weights row by row, each printed "%f " on one line. */
int lpaici_kernelset_write_text(const lpaici_kernelset *ks, const char *path);

int lpaici_kernelset_destroy(lpaici_kernelset *ks);

int lpaici_kernelset_get_info(const lpaici_kernelset *ks, lpaici_kernelset_info_t *info);

/* Copies out the dense cropped kernels (arrays sized dense_size and D*S), as the reference's
 * loader returns them (src/v1_0_lpa_ici_2D_fused.cpp:466-551). */
int lpaici_kernelset_get_dense(const lpaici_kernelset *ks, float *weights, int *offsets, int *rows, int *cols);

/* Copies out the run-length packing in the reference's layout (build_sparse_kernels,
 * src/v4_1_lpa_ici_2D_sparse_shared.cu:826-877): weights[n_taps]; run_row, run_col, run_len
 * [n_runs] (centre-relative); kernel_first_run, kernel_num_runs, kernel_first_weight [D*S]. */
int lpaici_kernelset_get_runs(const lpaici_kernelset *ks, float *weights, int *run_row, int *run_col, int *run_len,
                              int *kernel_first_run, int *kernel_num_runs, int *kernel_first_weight);

/* var[k] = (sigma*sigma) * sum(w_k^2) in float, k = d*S + s
 * (compute_kernel_variances, src/v1_0_lpa_ici_2D_fused.cpp:691-717). */
int lpaici_kernel_variances(const lpaici_kernelset *ks, float sigma, float *var);

/* ---- forward (device pointers) -------------------------------------------------------------- */

/* Denoises one grayscale FP32 image: for every direction and pixel, the scale sweep of sparse
 * correlations (no flip, anchor rows/2, cols/2, zero padding), the ICI interval intersection with
 * early exit, and the 1/variance-weighted aggregation over directions, in one kernel launch.
 *   d_noisy     width x height floats, row pitch noisy_pitch floats (>= width)
 *   d_denoised  width x height floats, row pitch out_pitch floats; must not overlap d_noisy
 *   sigma       noise standard deviation on the 0-1 scale (> 0); var = sigma^2 * sum w^2
 *   gamma       ICI threshold factor (> 0); interval = estimate -+ gamma*sqrt(var)
 *   d_scale_map optional (NULL): D*height*width bytes, direction-major, the index of the last
 *               accepted scale of every direction and pixel
 * Replaces the directional loop of anisotropic_lpa_ici_gpu_fused
 * (src/v4_1_lpa_ici_2D_sparse_shared.cu:1216-1235: 16 launches of process_direction_fused_kernel
 * :1007-1092, accumulate_direction_kernel :1104-1111 and normalize_estimate_kernel :1113-1120). */
int lpaici_forward(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                   int out_pitch, int width, int height, float sigma, float gamma, uint8_t *d_scale_map,
                   lpaici_stream_t stream);

/* lpaici_forward with every tap computed as one fused multiply-add (product and sum rounded once)
 * instead of a separately rounded product and sum: faster, and NOT bit-exact with the reference,
 * whose CPU build rounds both.  The selected scales can differ where an interval test is a tie at
 * FP32 rounding, which moves that pixel's output by up to about 1e-2 (4096^2 benchmark image: 70 of
 * 16.8 M pixels carry a flipped scale, 64 move by more than 1e-4, at most 1.07e-2); everywhere else the output differs from lpaici_forward's by a few ULP.  Same arguments and errors as
 * lpaici_forward.  No counterpart in the reference (whose GPU builds let the compiler contract some of
 * its multiply-adds). */
int lpaici_forward_ffma(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                        int out_pitch, int width, int height, float sigma, float gamma, uint8_t *d_scale_map,
                        lpaici_stream_t stream);

/* As lpaici_forward, with the per-kernel variances given by the caller (host array, D*S floats)
 * instead of sigma, as the reference's engine receives them (host_kernel_variances,
 * src/v4_1_lpa_ici_2D_sparse_shared.cu:1131). */
int lpaici_forward_var(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                       int out_pitch, int width, int height, const float *host_var, float gamma,
                       uint8_t *d_scale_map, lpaici_stream_t stream);

/* Row band of a larger image, for splitting one image across GPUs: d_in holds in_height rows of
 * the image (width columns, pitch in_pitch) and output row r of the band is input row
 * row_begin + r, for r < row_count.  Rows outside d_in are zero, so a band that carries `radius`
 * real rows above and below (or reaches the image border) gives exactly the full-image result.
 * d_scale_map, if not NULL, is D*row_count*width bytes. */
int lpaici_forward_rows(const lpaici_kernelset *ks, const float *d_in, int in_pitch, int width, int in_height,
                        int row_begin, int row_count, float *d_out, int out_pitch, float sigma, float gamma,
                        uint8_t *d_scale_map, lpaici_stream_t stream);

/* An image of `channels` interleaved channels (pixel x of row y, channel c at float y * pitch +
 * x * channels + c; pitches in floats, >= width * channels), every channel denoised on its own with
 * the same sigma and gamma, read and written in place with element stride `channels`.  The
 * reference's engine takes a channel count but implements one channel (its main converts every
 * image to gray); here channel c of the result equals the single-channel forward of channel c. */
int lpaici_forward_channels(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                            int out_pitch, int width, int height, int channels, float sigma, float gamma,
                            lpaici_stream_t stream);

/* ---- batched forward: images of uneven sizes, sigmas and gammas in one launch ---------------- */
typedef struct {
    const float *noisy;  /* device, width x height, pitch noisy_pitch floats */
    float *denoised;     /* device, width x height, pitch out_pitch floats */
    int width, height, noisy_pitch, out_pitch;
    float sigma, gamma;
    uint8_t *scale_map;  /* optional device D*height*width bytes, or NULL */
} lpaici_image;

typedef struct {
    int use_graph;   /* nonzero: capture the launch sequence in a CUDA graph at plan time, replay on run */
    int tile_config; /* -1: the configuration expected fastest for these images (per-tile times, autotuned
                      * or built in, times the waves of the whole tile queue); else an index
                      * < lpaici_num_tile_configs() */
} lpaici_batch_options;

typedef struct lpaici_batch lpaici_batch;

/* Plans a batch: orders all images' tiles largest-work-first into one work queue, uploads the
 * per-image descriptors (pointers, sizes, variances, thresholds) to device memory owned by the plan
 * and, with use_graph, captures the launch on `stream`.  The image pointers are baked in: rerun
 * the plan whenever their contents change, re-plan when the pointers change.  A plan of one image,
 * or of up to 64 images that share size, pitches, sigma and gamma, launches the single-image kernel
 * instead (one grid layer per image, no queue); the results are the same bit for bit.  No reference
 * counterpart (the reference denoises one image per process). */
int lpaici_batch_create(const lpaici_kernelset *ks, const lpaici_image *images, int n,
                        const lpaici_batch_options *opts, lpaici_stream_t stream, lpaici_batch **out);
int lpaici_batch_run(lpaici_batch *b, lpaici_stream_t stream);
int lpaici_batch_destroy(lpaici_batch *b);

/* One-shot: plan, run and free (synchronises the stream before freeing). */
int lpaici_forward_batched(const lpaici_kernelset *ks, const lpaici_image *images, int n, lpaici_stream_t stream);

/* Tile configurations the batched and single-image kernels can use. */
int lpaici_num_tile_configs(void);
int lpaici_tile_config_desc(int index, int *tile_w, int *tile_h, int *threads, int *pixels_per_thread);

/* Autotuner: times every tile configuration (one warm-up and `reps` timed launches each, CUDA
 * events on `stream`) on the device image d_sample (width x height, pitch floats) -- or, when
 * d_sample is NULL, on a built-in synthetic image of that size -- and makes the fastest the
 * default of this kernel set on the current device.  Per-configuration milliseconds go to
 * ms_out[lpaici_num_tile_configs()] when not NULL.  Synchronises `stream`. */
int lpaici_autotune(lpaici_kernelset *ks, const float *d_sample, int width, int height, int pitch, float sigma,
                    float gamma, int reps, int *best_config, float *ms_out, lpaici_stream_t stream);
/* Sets (config >= 0) or clears (config = -1) the default tile configuration of ks on the current device. */
int lpaici_set_tile_config(lpaici_kernelset *ks, int config);

/* ---- adjoint ---------------------------------------------------------------------------------- */

/* Gradient of L = sum_p g[p] * denoised[p] with respect to the noisy input, the ICI-selected scales
 * held fixed: grad[q] = sum_d sum_p g[p] * alpha_d(p) * h_{d,s*(d,p)}(q - p + c), with
 * alpha_d(p) = (1/v_d(p)) / sum_d' (1/v_d'(p)).  The selected scales and den are recomputed by an
 * exact forward sweep into a transient workspace (D*width*height bytes + 4*width*height bytes), taken
 * stream-ordered on `stream` from a memory pool this library owns on each device; the pool keeps freed
 * memory for later calls (lpaici_trim_workspace returns it).  The forward keeps nothing for the
 * adjoint.  No counterpart in the reference.
 *   d_grad_out  g, width x height (pitch gout_pitch);  d_grad_in  width x height (pitch gin_pitch) */
int lpaici_backward(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, const float *d_grad_out,
                    int gout_pitch, float *d_grad_in, int gin_pitch, int width, int height, float sigma,
                    float gamma, lpaici_stream_t stream);

/* Kept state, for callers that run the forward and then its adjoint (a training step) and can hold
 * D + 4 bytes per pixel: lpaici_forward_state is lpaici_forward (same output, bit for bit) that also
 * stores the selected scales and 1/den in caller-owned device memory d_state of
 * lpaici_adjoint_state_bytes(ks, width, height) bytes; lpaici_backward_state then runs the adjoint's
 * gather only (no selection pass), with the same sigma, and gives lpaici_backward's gradient bit for
 * bit.  lpaici_backward itself keeps nothing and recomputes the selection.  No counterpart in the
 * reference. */
size_t lpaici_adjoint_state_bytes(const lpaici_kernelset *ks, int width, int height);
int lpaici_forward_state(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch, float *d_denoised,
                         int out_pitch, int width, int height, float sigma, float gamma, void *d_state,
                         lpaici_stream_t stream);
int lpaici_backward_state(const lpaici_kernelset *ks, const void *d_state, const float *d_grad_out, int gout_pitch,
                          float *d_grad_in, int gin_pitch, int width, int height, float sigma,
                          lpaici_stream_t stream);

/* One image of a batched adjoint: noisy input, cotangent g and the gradient's buffer (device pointers,
 * pitches in floats), with the image's sigma and gamma. */
typedef struct {
    const float *noisy;
    const float *grad_out;
    float *grad_in;
    int width, height;
    int noisy_pitch, gout_pitch, gin_pitch;
    float sigma, gamma;
} lpaici_grad_image;

typedef struct lpaici_backward_batch lpaici_backward_batch;

/* Plans the adjoint of many images: pass A (selection) as one launch over all images'
 * tiles (the forward batch kernel writing s* and 1/den into memory the plan owns, D+4 bytes per
 * pixel), u = g/den over the plan's 1/den maps as one elementwise launch, pass B (gather) as one launch
 * over all images' tiles; with use_graph all three are captured in one CUDA graph.  Gradients equal lpaici_backward's, image by image, bit for bit.  The pointers are
 * baked in: rerun when the contents change, re-plan when the pointers change.  No counterpart in the
 * reference. */
int lpaici_backward_batch_create(const lpaici_kernelset *ks, const lpaici_grad_image *images, int n,
                                 const lpaici_batch_options *opts, lpaici_stream_t stream,
                                 lpaici_backward_batch **out);
int lpaici_backward_batch_run(lpaici_backward_batch *b, lpaici_stream_t stream);
int lpaici_backward_batch_destroy(lpaici_backward_batch *b);

/* Returns the memory cached in the adjoint's workspace pool on the current device to the driver. */
int lpaici_trim_workspace(void);

/* Size of the static device scratch behind lpaici_backward_noalloc: 64 MiB per device. */
#define LPAICI_NOALLOC_SCRATCH_BYTES (64u << 20)

/* lpaici_backward without any device allocation: same arguments and result (same kernels, so equal to
 * it), with its workspace and both kernel blobs in one file-scope __device__ array of
 * LPAICI_NOALLOC_SCRATCH_BYTES instead of the workspace pool and cudaMalloc.  For callers that cannot
 * allocate device memory during a step: a framework whose caching allocator already holds the free
 * memory, a loop that must not allocate after its setup, a device without stream-ordered memory
 * pools.  No counterpart in the reference.
 *   - Size limit: 256-byte-rounded (blob + mirrored blob + D*width*height bytes) + 4*width*height bytes
 *     must fit the scratch (with 16 directions about 3.3 Mpx, e.g. 1920 x 1080); larger images return
 *     LPAICI_ERR_UNSUPPORTED before any CUDA call.
 *   - Nothing has to start at zero: every call copies the blobs in (host to device on `stream`) and
 *     the selection sweep writes every byte the gather reads.
 *   - Every call looks up the array's address with cudaGetSymbolAddress; the first call on a device
 *     can load the module holding it, so a caller that captures streams makes that first call before.
 *   - Under CUDA's default lazy module loading, the 64 MiB are reserved on a device only once a process
 *     calls this entry point there; with CUDA_MODULE_LOADING=EAGER every process that loads the
 *     library reserves them on every device it uses, forward-only and command-line users included.
 *   - One scratch per device: calls that overlap on one device (different streams or threads with
 *     work in flight at once) race on it.  Serialise them, e.g. on one stream. */
int lpaici_backward_noalloc(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch,
                            const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch, int width,
                            int height, float sigma, float gamma, lpaici_stream_t stream);

/* ---- host-pointer entry points ---------------------------------------------------------------- */

/* The reference engine's own signature and ownership (anisotropic_lpa_ici_gpu_fused,
 * src/v4_1_lpa_ici_2D_sparse_shared.cu:1122-1244): host input and output buffers, the dense
 * kernels and the caller's variances; copies in, denoises on the current device, copies out,
 * synchronously.  channels: 1, or up to 64 interleaved channels denoised one by one (the reference
 * implements one; lpaici_forward_channels); host_global_weights_buffer is unused (may be NULL), as on the
 * reference's GPU path.  *seconds, if not NULL, receives the reference's timing window: from
 * after the uploads to after the copy of the result back to the host (:1216-1240).
 * Errors are returned instead of exiting the process. */
int lpaici_anisotropic_gpu_fused(float *host_img_noisy, float *host_img_denoised, int width, int height,
                                 int channels, float *host_global_weights_buffer, int num_dirs, int num_scales,
                                 float *host_kernel_weights, int host_kernel_weights_size, int *host_offsets,
                                 int *host_rows, int *host_cols, float *host_kernel_variances, float ici_gamma,
                                 double *seconds);

/* Kernel-set form of the above: host in, host out, sigma/gamma, through device buffers cached
 * per thread and device (grown on demand, never shrunk; lpaici_release_host_buffers frees them).
 * The image goes through in row bands: the upload of a band's rows, its forward and its download
 * run on separate streams, so with pinned host buffers the copies overlap the kernels; the result
 * equals one full-image launch bit for bit.  Ordered after earlier work on `stream`; returns when
 * the output is in host memory. */
int lpaici_denoise_host(const lpaici_kernelset *ks, const float *host_noisy, float *host_denoised, int width,
                        int height, float sigma, float gamma, lpaici_stream_t stream);
int lpaici_release_host_buffers(void);

/* ---- reference utilities (host) ---------------------------------------------------------------- */

/* noisy[i] = clean[i] + N(0, sigma) drawn from std::mt19937{seed} and
 * std::normal_distribution<float>{0, sigma}, one sample per pixel in order
 * (create_noisy_image, src/v1_0_lpa_ici_2D_fused.cpp:759-776). */
int lpaici_add_noise(const float *clean, float *noisy, long n, float sigma, unsigned int seed);

/* 10*log10(1/MSE), squared float differences summed in double
 * (calculate_PSNR, src/v1_0_lpa_ici_2D_fused.cpp:778-799). */
double lpaici_psnr(const float *a, const float *b, long n);

#ifdef __cplusplus
}
#endif
#endif /* LPAICI_H */
