// batched.cu -- many images of uneven sizes, sigmas and gammas in one launch.
//
// The plan cuts every image into the tiles of one tile configuration and orders the tiles into a
// single work queue, full tiles of the largest images first and partial edge tiles last, so the
// cheap ragged tiles fill the tail.  The launch has one CTA per queue item: the hardware dispatches
// blocks in index order as SMs free up, so the queue order is the execution order without a
// persistent loop (measured: a persistent grid pulling items from an atomic counter kept its
// 768-thread instances at the 80-register limit and ran 2-2.5 % slower).  There is no inter-CTA
// waiting of any kind.  With use_graph the launch is captured once into a CUDA graph and replayed
// by lpaici_batch_run.  A plan of one image launches the single-image kernel instead (image and tables
// as launch parameters): there are no small-image tails to fill, and the queue decode would cost a
// little per CTA.  A plan of up to kMaxMultiImages images of one size, pitch, sigma and gamma launches
// that kernel once with a grid layer per image (lpaici_forward_multi_kernel).
// No reference counterpart: the reference denoises one image per process
// (src/v4_1_lpa_ici_2D_sparse_shared.cu:365-530).
#include <algorithm>
#include <cstring>
#include <vector>

#include "configs.h"
#include "tile_core.cuh"

namespace lpaici {

// Per-image descriptor in device memory.
struct BatchImage {
    const float *in;
    float *out;       // null: no estimate (the adjoint's selection pass)
    uint8_t *smap;
    float *rden;      // optional 1/den map (the adjoint's selection pass)
    int W, H, in_pitch, out_pitch;
    int tab_offset;  // float index of var[nk] (thr[nk] follows) in the plan's table array
    int pad;
};

struct BatchArgs {
    const BatchImage *images;
    const float *tables;    // per image var[nk], thr[nk]
    const int2 *items;      // (image, tile index within the image)
    int n_items;
    int D, S, R;
    const int *blob;
    int blob_words, run_word, weight_word;
    float neg_zero;  // -0.0f, read at run time (see prod2 in tile_core.cuh)
    // every image of the plan has the same sigma and gamma (always so for one image): its var and thr
    // travel here, as in the single-image launch, instead of being read per CTA from `tables`
    int shared_tables;
    float var[kMaxKernels];
    float thr[kMaxKernels];
};

template <int WX, int WY, int Q>
__global__ void __launch_bounds__(32 * WX * WY, 1)
    lpaici_batched_kernel(const __grid_constant__ BatchArgs a) {
    using Shape = TileShape<WX, WY, Q>;
    extern __shared__ __align__(16) int smem[];
    const int nk = a.D * a.S;
    int *s_blob = smem;
    float *s_tab = reinterpret_cast<float *>(smem + a.blob_words);
    float2 *s_tile = reinterpret_cast<float2 *>(smem + a.blob_words + table_words(nk));
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, a.R, Q);

    // the CTA's image arguments live in shared memory: in registers they would stay live across the
    // whole sweep, beside the run loop's (the single-image kernel reads them from its parameters)
    __shared__ __align__(16) unsigned char s_img_raw[sizeof(ImageArgs)];
    __shared__ int2 s_xy;
    ImageArgs &s_img = *reinterpret_cast<ImageArgs *>(s_img_raw);
    const int item = blockIdx.x;  // one CTA per queue item, dispatched in queue order
    if (item >= a.n_items) return;
    if (threadIdx.x == 0) {
        const int2 it = a.items[item];
        const BatchImage bi = a.images[it.x];
        const int tiles_x = (bi.W + Shape::kTileW - 1) / Shape::kTileW;
        ImageArgs img{};
        img.in = bi.in;
        img.out = bi.out;
        img.smap = bi.smap;
        img.rden = bi.rden;
        img.W = bi.W;
        img.in_h = bi.H;
        img.in_pitch = bi.in_pitch;
        img.out_pitch = bi.out_pitch;
        img.row_begin = 0;
        img.rows_out = bi.H;
        s_img = img;
        s_xy = make_int2((it.y % tiles_x) * Shape::kTileW, (it.y / tiles_x) * Shape::kTileH);
    }
    stage_blob(s_blob, a.blob, a.blob_words, a.run_word, a.weight_word, g.pitch2);
    if (a.shared_tables) stage_tables(s_tab, a.var, a.thr, nk);
    __syncthreads();
    if (!a.shared_tables) {
        const float *t = a.tables + a.images[a.items[item].x].tab_offset;
        stage_tables(s_tab, t, t + nk, nk);
    }
    const int x0 = s_xy.x, y0 = s_xy.y;
    load_tile(s_tile, s_img, x0, y0, g);
    __syncthreads();
    sweep_tile<WX, Q>(s_img, x0, y0, a.D, a.S, g, s_blob, a.run_word, a.weight_word, s_tab, s_tile, a.neg_zero);
}

namespace {

struct KernelInfo {
    const void *fn;
    int tile_w, tile_h, threads;
    size_t smem;
};

template <int WX, int WY, int Q>
int batched_info(const KernelTables &tab, KernelInfo *info) {
    using Shape = TileShape<WX, WY, Q>;
    const TileGeom g = TileGeom::make(Shape::kTileW, Shape::kTileH, tab.R, Q);
    const int nk = tab.D * tab.S;
    info->fn = reinterpret_cast<const void *>(lpaici_batched_kernel<WX, WY, Q>);
    info->tile_w = Shape::kTileW;
    info->tile_h = Shape::kTileH;
    info->threads = Shape::kThreads;
    info->smem = sizeof(int) * (tab.blob_words + table_words(nk)) + g.tile_bytes();
    return LPAICI_OK;
}

int get_info(int config, const KernelTables &tab, KernelInfo *info) {
#define LPAICI_BATCH_CASE(idx, WX, WY, Q) \
    case idx: return batched_info<WX, WY, Q>(tab, info);
    switch (config) {
        LPAICI_TILE_CONFIGS(LPAICI_BATCH_CASE)
        default: return set_error(LPAICI_ERR_INVALID_ARG, "tile config %d out of range", config);
    }
#undef LPAICI_BATCH_CASE
}

}  // namespace
}  // namespace lpaici

using namespace lpaici;

struct lpaici_batch {
    int device = -1;
    KernelInfo info{};
    BatchArgs args{};
    int grid = 0;
    void *dev_mem = nullptr;  // images | tables | items
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // a plan of one image runs the single-image kernel (image and tables as launch parameters, no queue
    // to decode): one image has no small-image tails for the queue to fill
    bool single = false;
    // a plan of 2 .. kMaxMultiImages images of one size, pitch, sigma and gamma runs the single-image kernel
    // once with a grid layer per image (lpaici_forward_multi_kernel): no queue to decode, and each image's
    // CTAs fill the SMs the previous image's last wave leaves idle
    bool multi = false;
    int n_multi = 0;
    MultiImages mi{};
    ImageArgs img{};
    KernelTables tab{};
    int config = 0;
};

namespace lpaici {

int batch_plan_enqueue(lpaici_batch *b, cudaStream_t stream) {
    if (b->single) return launch_forward(nullptr, b->img, b->tab, b->config, stream);
    if (b->multi) return launch_forward_multi(b->img, b->tab, b->mi, b->n_multi, b->config, stream);
    void *params[] = {&b->args};
    const cudaError_t e = cudaLaunchKernel(b->info.fn, dim3(b->grid), dim3(b->info.threads), params, b->info.smem, stream);
    if (e != cudaSuccess) return cuda_error(e, "batched launch");
    return LPAICI_OK;
}

void batch_plan_free(lpaici_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->dev_mem) cudaFree(b->dev_mem);
    delete b;
}

// The plan of lpaici_batch_create for already validated images (specs); the adjoint's batched
// selection pass uses it with out = null and smap/rden set.
int batch_plan_create(const lpaici_kernelset *ks, const BatchSpec *specs, int n, int config, bool use_graph,
                      cudaStream_t stream, lpaici_batch **out) {
    *out = nullptr;
    const int nk = ks->D * ks->S;
    if (ks->S > kMaxScales)
        return set_error(LPAICI_ERR_UNSUPPORTED, "%d scales per direction; the kernels support at most %d", ks->S,
                         kMaxScales);
    const int *blob = nullptr;
    int rc = device_blob(ks, &blob);
    if (rc != LPAICI_OK) return rc;

    auto *b = new lpaici_batch();
    cudaGetDevice(&b->device);
    KernelTables tab;
    fill_tables(ks, nullptr, 1.0f, 1.0f, &tab);
    tab.blob = blob;
    rc = get_info(config, tab, &b->info);
    if (rc != LPAICI_OK) {
        batch_plan_free(b);
        return rc;
    }

    // host images: descriptors, tables, and the ordered work queue
    std::vector<BatchImage> imgs(n);
    std::vector<float> tables(static_cast<size_t>(n) * 2 * nk);
    struct Item {
        int image, tile;
        long key;
    };
    std::vector<Item> items;
    for (int i = 0; i < n; i++) {
        const BatchSpec &im = specs[i];
        KernelTables t;
        fill_tables(ks, nullptr, im.sigma, im.gamma, &t);
        std::memcpy(&tables[static_cast<size_t>(i) * 2 * nk], t.var, sizeof(float) * nk);
        std::memcpy(&tables[static_cast<size_t>(i) * 2 * nk + nk], t.thr, sizeof(float) * nk);
        imgs[i] = BatchImage{im.noisy, im.out, im.smap, im.rden, im.width, im.height, im.noisy_pitch, im.out_pitch,
                             i * 2 * nk, 0};
        const int tx = (im.width + b->info.tile_w - 1) / b->info.tile_w;
        const int ty = (im.height + b->info.tile_h - 1) / b->info.tile_h;
        const long area = static_cast<long>(im.width) * im.height;
        for (int y = 0; y < ty; y++)
            for (int x = 0; x < tx; x++) {
                const int w = std::min(b->info.tile_w, im.width - x * b->info.tile_w);
                const int h = std::min(b->info.tile_h, im.height - y * b->info.tile_h);
                // full tiles first, then by image size (largest first), then raster order
                items.push_back({i, y * tx + x, static_cast<long>(w) * h * (1L << 40) + area});
            }
    }
    std::stable_sort(items.begin(), items.end(), [](const Item &p, const Item &q) { return p.key > q.key; });
    std::vector<int2> qitems(items.size());
    for (size_t j = 0; j < items.size(); j++) qitems[j] = make_int2(items[j].image, items[j].tile);

    const size_t img_bytes = sizeof(BatchImage) * n;
    const size_t tab_off = (img_bytes + 255) & ~size_t(255);
    const size_t tab_bytes = sizeof(float) * tables.size();
    const size_t item_off = (tab_off + tab_bytes + 255) & ~size_t(255);
    const size_t item_bytes = sizeof(int2) * qitems.size();
    const size_t total = item_off + item_bytes;
    cudaError_t e = cudaMalloc(&b->dev_mem, total);
    if (e != cudaSuccess) {
        batch_plan_free(b);
        return cuda_error(e, "cudaMalloc(batch plan)");
    }
    char *base = static_cast<char *>(b->dev_mem);
    e = cudaMemcpy(base, imgs.data(), img_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + tab_off, tables.data(), tab_bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(base + item_off, qitems.data(), item_bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        batch_plan_free(b);
        return cuda_error(e, "cudaMemcpy(batch plan)");
    }
    b->args.images = reinterpret_cast<const BatchImage *>(base);
    b->args.tables = reinterpret_cast<const float *>(base + tab_off);
    b->args.items = reinterpret_cast<const int2 *>(base + item_off);
    b->args.n_items = static_cast<int>(qitems.size());
    b->args.D = ks->D;
    b->args.S = ks->S;
    b->args.R = ks->radius;
    b->args.blob = blob;
    b->args.blob_words = tab.blob_words;
    b->args.run_word = tab.run_word;
    b->args.weight_word = tab.weight_word;
    b->args.neg_zero = -0.0f;
    bool same = true;
    for (int i = 1; i < n; i++) same = same && specs[i].sigma == specs[0].sigma && specs[i].gamma == specs[0].gamma;
    b->args.shared_tables = same ? 1 : 0;
    if (same) {
        std::memcpy(b->args.var, tables.data(), sizeof(float) * nk);
        std::memcpy(b->args.thr, tables.data() + nk, sizeof(float) * nk);
    }

    int max_optin = 0, per_sm = 0;
    cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
    if (b->info.smem > static_cast<size_t>(max_optin)) {
        batch_plan_free(b);
        return set_error(LPAICI_ERR_UNSUPPORTED, "batched tile needs %zu B of shared memory, device allows %d",
                         b->info.smem, max_optin);
    }
    e = cudaFuncSetAttribute(b->info.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(b->info.smem));
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, b->info.fn, b->info.threads, b->info.smem);
    if (e != cudaSuccess || per_sm <= 0) {
        batch_plan_free(b);
        return e != cudaSuccess ? cuda_error(e, "batched occupancy")
                                : set_error(LPAICI_ERR_UNSUPPORTED, "batched kernel does not fit on an SM");
    }
    b->grid = b->args.n_items;  // one CTA per queue item
    bool one_size = n >= 2 && n <= kMaxMultiImages;
    for (int i = 1; one_size && i < n; i++) {
        const BatchSpec &a0 = specs[0], &ai = specs[i];
        one_size = ai.width == a0.width && ai.height == a0.height && ai.noisy_pitch == a0.noisy_pitch &&
                   ai.out_pitch == a0.out_pitch && ai.sigma == a0.sigma && ai.gamma == a0.gamma &&
                   (ai.out == nullptr) == (a0.out == nullptr) && (ai.smap == nullptr) == (a0.smap == nullptr) &&
                   (ai.rden == nullptr) == (a0.rden == nullptr);
    }
    if (n == 1 || one_size) {
        const BatchSpec &im = specs[0];
        b->single = n == 1;
        b->multi = one_size;
        b->n_multi = one_size ? n : 0;
        for (int i = 0; one_size && i < n; i++) {
            b->mi.in[i] = specs[i].noisy;
            b->mi.out[i] = specs[i].out;
            b->mi.smap[i] = specs[i].smap;
            b->mi.rden[i] = specs[i].rden;
        }
        b->config = config;
        b->img.in = im.noisy;
        b->img.out = im.out;
        b->img.smap = im.smap;
        b->img.rden = im.rden;
        b->img.W = im.width;
        b->img.in_h = im.height;
        b->img.in_pitch = im.noisy_pitch;
        b->img.out_pitch = im.out_pitch;
        b->img.row_begin = 0;
        b->img.rows_out = im.height;
        fill_tables(ks, nullptr, im.sigma, im.gamma, &b->tab);
        b->tab.blob = blob;
    }

    b->use_graph = use_graph;
    if (b->use_graph) {
        cudaStream_t cap = nullptr;
        e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = batch_plan_enqueue(b, cap);
            cudaError_t e2 = cudaStreamEndCapture(cap, &b->graph);
            if (rc == LPAICI_OK && e2 != cudaSuccess) rc = cuda_error(e2, "cudaStreamEndCapture");
            if (rc == LPAICI_OK) {
                e = cudaGraphInstantiate(&b->exec, b->graph, 0);
                if (e != cudaSuccess) rc = cuda_error(e, "cudaGraphInstantiate");
            }
        } else {
            rc = cuda_error(e, "graph capture");
        }
        if (cap) cudaStreamDestroy(cap);
        if (rc != LPAICI_OK) {
            batch_plan_free(b);
            return rc;
        }
        e = cudaGraphUpload(b->exec, stream);
        if (e != cudaSuccess) {
            batch_plan_free(b);
            return cuda_error(e, "cudaGraphUpload");
        }
    }
    *out = b;
    return LPAICI_OK;
}

}  // namespace lpaici

extern "C" {

int lpaici_batch_create(const lpaici_kernelset *ks, const lpaici_image *images, int n, const lpaici_batch_options *opts,
                        lpaici_stream_t stream_, lpaici_batch **out) {
    if (!ks || !images || n <= 0 || !out) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_batch_create: bad argument");
    *out = nullptr;
    std::vector<BatchSpec> specs(n);
    for (int i = 0; i < n; i++) {
        const lpaici_image &im = images[i];
        if (!im.noisy || !im.denoised || im.width <= 0 || im.height <= 0 || im.noisy_pitch < im.width ||
            im.out_pitch < im.width)
            return set_error(LPAICI_ERR_INVALID_ARG, "batch image %d: bad pointer or size", i);
        if (!(im.sigma > 0.0f) || !(im.gamma > 0.0f))
            return set_error(LPAICI_ERR_INVALID_ARG, "batch image %d: sigma and gamma need positive numbers", i);
        specs[i] = BatchSpec{im.noisy, im.denoised, im.scale_map, nullptr, im.width, im.height, im.noisy_pitch,
                             im.out_pitch, im.sigma, im.gamma};
    }
    int config = opts ? opts->tile_config : -1;
    if (config < 0) {
        std::vector<int> w(n), h(n);
        for (int i = 0; i < n; i++) {
            w[i] = specs[i].width;
            h[i] = specs[i].height;
        }
        config = config_for_images(ks, w.data(), h.data(), n);
    }
    return batch_plan_create(ks, specs.data(), n, config, opts && opts->use_graph,
                             reinterpret_cast<cudaStream_t>(stream_), out);
}

int lpaici_batch_run(lpaici_batch *b, lpaici_stream_t stream_) {
    if (!b) return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_batch_run: null plan");
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != b->device)
        return set_error(LPAICI_ERR_INVALID_ARG, "batch planned on device %d, current device is %d", b->device, dev);
    if (b->use_graph) {
        cudaError_t e = cudaGraphLaunch(b->exec, stream);
        if (e != cudaSuccess) return cuda_error(e, "cudaGraphLaunch");
        return LPAICI_OK;
    }
    return batch_plan_enqueue(b, stream);
}

int lpaici_batch_destroy(lpaici_batch *b) {
    if (b) {
        int cur = -1;
        cudaGetDevice(&cur);
        cudaSetDevice(b->device);
        cudaDeviceSynchronize();
        batch_plan_free(b);
        if (cur >= 0) cudaSetDevice(cur);
    }
    return LPAICI_OK;
}

int lpaici_forward_batched(const lpaici_kernelset *ks, const lpaici_image *images, int n, lpaici_stream_t stream) {
    lpaici_batch *b = nullptr;
    lpaici_batch_options opts{0, -1};
    int rc = lpaici_batch_create(ks, images, n, &opts, stream, &b);
    if (rc != LPAICI_OK) return rc;
    rc = lpaici_batch_run(b, stream);
    cudaError_t e = cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream));
    if (rc == LPAICI_OK && e != cudaSuccess) rc = cuda_error(e, "cudaStreamSynchronize");
    batch_plan_free(b);
    return rc;
}

}  // extern "C"
