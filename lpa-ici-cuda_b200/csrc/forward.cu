// forward.cu -- single-image LPA-ICI forward: one launch, one CTA per output tile, all directions
// and scales of the tile inside the CTA, aggregation in registers.
//
// Replaces the directional loop of anisotropic_lpa_ici_gpu_fused
// (src/v4_1_lpa_ici_2D_sparse_shared.cu:1216-1235), i.e. 16 launches of
// process_direction_fused_kernel (:1007-1092) + accumulate_direction_kernel (:1104-1111) and one
// normalize_estimate_kernel (:1113-1120), with the kernel set read from global memory (staged in
// shared memory per CTA) instead of capacity-limited constant memory.
#include "tile_core.cuh"
#include "configs.h"

namespace lpaici {

// Fused = false: every tap's product and sum rounded on their own (bit-exact with the reference);
// true: each tap one fused multiply-add (lpaici_forward_ffma).
template <int WX, int WY, int Q, bool Fused>
__global__ void __launch_bounds__(32 * WX * WY, 1)
    lpaici_forward_kernel(const __grid_constant__ ImageArgs img, const __grid_constant__ KernelTables tab) {
    using Shape = TileShape<WX, WY, Q>;
    extern __shared__ __align__(16) int smem[];
    const int nk = tab.D * tab.S;
    int *s_blob = smem;
    float *s_tab = reinterpret_cast<float *>(smem + tab.blob_words);
    float2 *s_tile = reinterpret_cast<float2 *>(smem + tab.blob_words + table_words(nk));
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R, Q);
    const int x0 = blockIdx.x * Shape::kTileW, y0 = blockIdx.y * Shape::kTileH;

    stage_blob(s_blob, tab.blob, tab.blob_words, tab.run_word, tab.weight_word, g.pitch2);
    stage_tables(s_tab, tab.var, tab.thr, nk);
    load_tile(s_tile, img, x0, y0, g);
    __syncthreads();
    sweep_tile<WX, Q, Fused>(img, x0, y0, tab.D, tab.S, g, s_blob, tab.run_word, tab.weight_word, s_tab, s_tile,
                             tab.neg_zero);
}

// Several images of one size, pitch, sigma and gamma in one launch (a batched plan of such images):
// grid layer z is image z, whose buffers replace img's; everything else is the single-image kernel.  The
// CTAs of image z + 1 fill the SMs image z's last wave leaves idle.  No counterpart in the reference.
template <int WX, int WY, int Q>
__global__ void __launch_bounds__(32 * WX * WY, 1)
    lpaici_forward_multi_kernel(const __grid_constant__ ImageArgs img, const __grid_constant__ KernelTables tab,
                                const __grid_constant__ MultiImages mi) {
    using Shape = TileShape<WX, WY, Q>;
    extern __shared__ __align__(16) int smem[];
    const int nk = tab.D * tab.S;
    int *s_blob = smem;
    float *s_tab = reinterpret_cast<float *>(smem + tab.blob_words);
    float2 *s_tile = reinterpret_cast<float2 *>(smem + tab.blob_words + table_words(nk));
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R, Q);
    const int x0 = blockIdx.x * Shape::kTileW, y0 = blockIdx.y * Shape::kTileH;
    ImageArgs im = img;
    im.in = mi.in[blockIdx.z];
    im.out = mi.out[blockIdx.z];
    im.smap = mi.smap[blockIdx.z];
    im.rden = mi.rden[blockIdx.z];

    stage_blob(s_blob, tab.blob, tab.blob_words, tab.run_word, tab.weight_word, g.pitch2);
    stage_tables(s_tab, tab.var, tab.thr, nk);
    load_tile(s_tile, im, x0, y0, g);
    __syncthreads();
    sweep_tile<WX, Q, false>(im, x0, y0, tab.D, tab.S, g, s_blob, tab.run_word, tab.weight_word, s_tab, s_tile,
                             tab.neg_zero);
}

namespace {

template <int WX, int WY, int Q>
int launch_multi_cfg(const ImageArgs &img, const KernelTables &tab, const MultiImages &mi, int n,
                     cudaStream_t stream) {
    using Shape = TileShape<WX, WY, Q>;
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R, Q);
    const int nk = tab.D * tab.S;
    const size_t smem = sizeof(int) * (tab.blob_words + table_words(nk)) + g.tile_bytes();
    auto kern = lpaici_forward_multi_kernel<WX, WY, Q>;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > static_cast<size_t>(max_optin))
        return set_error(LPAICI_ERR_UNSUPPORTED, "forward tile needs %zu B of shared memory, device allows %d", smem,
                         max_optin);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(forward, several images)");
    const dim3 grid((img.W + Shape::kTileW - 1) / Shape::kTileW, (img.rows_out + Shape::kTileH - 1) / Shape::kTileH,
                    n);
    if (grid.y > 65535u) return set_error(LPAICI_ERR_UNSUPPORTED, "image too tall: %d rows", img.rows_out);
    kern<<<grid, Shape::kThreads, smem, stream>>>(img, tab, mi);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "forward launch (several images)");
    return LPAICI_OK;
}

template <int WX, int WY, int Q, bool Fused>
int launch_cfg(const ImageArgs &img, const KernelTables &tab, cudaStream_t stream) {
    using Shape = TileShape<WX, WY, Q>;
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R, Q);
    const int nk = tab.D * tab.S;
    const size_t smem = sizeof(int) * (tab.blob_words + table_words(nk)) + g.tile_bytes();
    auto kern = lpaici_forward_kernel<WX, WY, Q, Fused>;
    int dev = 0, max_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > static_cast<size_t>(max_optin))
        return set_error(LPAICI_ERR_UNSUPPORTED, "forward tile needs %zu B of shared memory, device allows %d", smem,
                         max_optin);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute(forward)");
    const dim3 grid((img.W + Shape::kTileW - 1) / Shape::kTileW, (img.rows_out + Shape::kTileH - 1) / Shape::kTileH);
    if (grid.y > 65535u) return set_error(LPAICI_ERR_UNSUPPORTED, "image too tall: %d rows", img.rows_out);
    kern<<<grid, Shape::kThreads, smem, stream>>>(img, tab);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "forward launch");
    return LPAICI_OK;
}

}  // namespace

#define LPAICI_FWD_CASE(idx, WX, WY, Q) \
    case idx: return fused ? launch_cfg<WX, WY, Q, true>(img, tab, stream) : launch_cfg<WX, WY, Q, false>(img, tab, stream);

template <int WX, int WY, int Q>
int blocks_per_sm(size_t smem) {
    auto kern = lpaici_forward_kernel<WX, WY, Q, false>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, TileShape<WX, WY, Q>::kThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int config_blocks_per_sm(int config, size_t smem) {
#define LPAICI_BPS_CASE(idx, WX, WY, Q) \
    case idx: return blocks_per_sm<WX, WY, Q>(smem);
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_BPS_CASE)
        default: return 0;
    }
#undef LPAICI_BPS_CASE
}

void config_tile(int config, int *tile_w, int *tile_h) {
#define LPAICI_TILE_CASE(idx, WX, WY, Q) \
    case idx:                            \
        *tile_w = 4 * (Q) * (WX);        \
        *tile_h = 16 * (WY);             \
        return;
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_TILE_CASE)
        default: *tile_w = *tile_h = 1;
    }
#undef LPAICI_TILE_CASE
}

// Shared memory a tile configuration needs for a kernel set: blob + tables + the T8 tile.
size_t config_smem(int config, int blob_words, int nk, int R) {
#define LPAICI_SMEM_CASE(idx, WX, WY, Q)                                                   \
    case idx:                                                                              \
        return sizeof(int) * (blob_words + table_words(nk)) +                              \
               TileGeom::make(4 * (Q) * (WX), 16 * (WY), R, Q).tile_bytes();
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_SMEM_CASE)
        default: return ~size_t(0);
    }
#undef LPAICI_SMEM_CASE
}

int launch_forward_multi(const ImageArgs &img, const KernelTables &tab, const MultiImages &mi, int n, int config,
                         cudaStream_t stream) {
    if (tab.S > kMaxScales)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%d scales per direction; the kernels support at most %d", tab.S,
                         kMaxScales);
    if (n < 1 || n > kMaxMultiImages)
        return set_error(LPAICI_ERR_INVALID_ARG, "%d images in one launch; at most %d", n, kMaxMultiImages);
#define LPAICI_MULTI_CASE(idx, WX, WY, Q) \
    case idx: return launch_multi_cfg<WX, WY, Q>(img, tab, mi, n, stream);
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_MULTI_CASE)
        default: return set_error(LPAICI_ERR_INVALID_ARG, "tile config %d out of range", config);
    }
#undef LPAICI_MULTI_CASE
}

int launch_forward(const lpaici_kernelset *ks, const ImageArgs &img, const KernelTables &tab, int config,
                   cudaStream_t stream, bool fused) {
    (void)ks;
    if (tab.S > kMaxScales)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%d scales per direction; the kernels support at most %d", tab.S,
                         kMaxScales);
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_FWD_CASE)
        default: return set_error(LPAICI_ERR_INVALID_ARG, "tile config %d out of range", config);
    }
}

}  // namespace lpaici
