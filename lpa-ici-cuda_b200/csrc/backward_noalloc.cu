// backward_noalloc.cu -- lpaici_backward_noalloc: the adjoint of lpaici_backward with every transient
// buffer placed in one file-scope device array, so that a call allocates no device memory at all (no
// cudaMalloc, cudaMallocAsync or memory pool; no torch).
//
// Scratch layout (each part starts on a 256-byte boundary):
//   [forward kernel blob | mirrored kernel blob | D*W*H selection bytes | W*H floats of 1/den]
// Nothing in it needs to start at zero: the two blobs are copied in by every call, pass A writes every
// selection byte and 1/den value that pass B reads.
//
// The array lives in its own translation unit.  Under CUDA's default lazy module loading the module that
// holds it is loaded, and its 64 MiB reserved on a device, only when a process calls this entry point on
// that device; with CUDA_MODULE_LOADING=EAGER every process that loads the library reserves it on every
// device it uses.  No counterpart in the reference.

#include "internal.h"

using namespace lpaici;

namespace {

constexpr size_t kScratchBytes = LPAICI_NOALLOC_SCRATCH_BYTES;
__device__ __align__(256) unsigned char g_adjoint_scratch[kScratchBytes];

size_t round256(size_t n) { return (n + 255) & ~size_t(255); }

// Address of the scratch array on the current device.  Looked up on every call (cheap once the module
// is loaded): after a cudaDeviceReset the module is loaded again, possibly at another address.  In host
// code g_adjoint_scratch names a host-side stand-in, never a device address.  The first call on a
// device can load the module holding the array.
int scratch_address(unsigned char **out) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_adjoint_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(adjoint scratch)");
    *out = static_cast<unsigned char *>(p);
    return LPAICI_OK;
}

}  // namespace

extern "C" int lpaici_backward_noalloc(const lpaici_kernelset *ks, const float *d_noisy, int noisy_pitch,
                                       const float *d_grad_out, int gout_pitch, float *d_grad_in, int gin_pitch,
                                       int width, int height, float sigma, float gamma, lpaici_stream_t stream_) {
    if (!ks || !d_noisy || !d_grad_out || !d_grad_in)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward_noalloc: null argument");
    if (width <= 0 || height <= 0 || noisy_pitch < width || gout_pitch < width || gin_pitch < width)
        return set_error(LPAICI_ERR_INVALID_ARG, "lpaici_backward_noalloc: bad size or pitch");
    const int prc = check_adjoint_params(ks, sigma, &gamma, "lpaici_backward_noalloc");
    if (prc != LPAICI_OK) return prc;

    // sizes are checked before any CUDA call
    const size_t npx = static_cast<size_t>(width) * height;
    const size_t blob_bytes = round256(sizeof(int) * ks->blob.size());
    const size_t adj_bytes = round256(sizeof(int) * ks->adj_blob.size());
    const size_t smap_bytes = round256(static_cast<size_t>(ks->D) * npx);
    const size_t need = blob_bytes + adj_bytes + smap_bytes + sizeof(float) * npx;
    if (need > kScratchBytes)
        return set_error(LPAICI_ERR_UNSUPPORTED,
                         "lpaici_backward_noalloc: a %dx%d image with %d directions needs %zu bytes of scratch, the "
                         "static scratch holds %zu (LPAICI_NOALLOC_SCRATCH_BYTES); use lpaici_backward",
                         width, height, ks->D, need, kScratchBytes);

    unsigned char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != LPAICI_OK) return rc;
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    int *blob = reinterpret_cast<int *>(base);
    int *adj = reinterpret_cast<int *>(base + blob_bytes);
    uint8_t *smap = base + blob_bytes + adj_bytes;
    float *rden = reinterpret_cast<float *>(base + blob_bytes + adj_bytes + smap_bytes);
    cudaError_t e = cudaMemcpyAsync(blob, ks->blob.data(), sizeof(int) * ks->blob.size(), cudaMemcpyHostToDevice,
                                    stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(adj, ks->adj_blob.data(), sizeof(int) * ks->adj_blob.size(), cudaMemcpyHostToDevice,
                            stream);
    if (e != cudaSuccess) return cuda_error(e, "lpaici_backward_noalloc: kernel blobs to scratch");
    return adjoint_passes(ks, blob, adj, smap, rden, d_noisy, noisy_pitch, d_grad_out, gout_pitch, d_grad_in, gin_pitch,
                          width, height, sigma, gamma, stream);
}
