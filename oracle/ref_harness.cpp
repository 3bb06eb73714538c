// ref_harness.cpp -- builds one of the reference's CPU sources in-process.  TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file once per reference source (REF_SOURCE = the path of
// src/v1_0_lpa_ici_2D_fused.cpp or src/v0_0_lpa_ici_2D_naive.cpp of titocapovilla/lpa-ici-cuda,
// REF_ENGINE = anisotropic_lpa_ici_cpu_fused or anisotropic_lpa_ici_cpu_naive) with the reference's
// own flags (-std=c++17 -O3, no -march), renaming its main() so that the unmodified functions can be
// called from Python through the C wrappers below.  The output goes to oracle/_ref/ only.
//
// Nothing of the reference is copied: the source is #included from where it lies.
#define main lpaici_reference_main
#include REF_SOURCE
#undef main

#include <cstdlib>
#include <cstring>

template <typename T> static T *dup_vec(const std::vector<T> &v) {
    T *p = static_cast<T *>(std::malloc(sizeof(T) * (v.size() ? v.size() : 1)));
    if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

extern "C" {

// load_LPA_kernels_standardized (v1_0_lpa_ici_2D_fused.cpp:466-551); returns 1 on success.
int ref_load_kernels(const char *path, int *D, int *S, float **w, int *nw, int **off, int **rows, int **cols) {
    std::vector<float> hw;
    std::vector<int> ho, hr, hc;
    int d = 0, s = 0;
    if (!load_LPA_kernels_standardized(path, hw, ho, hr, hc, d, s)) return 0;
    *D = d;
    *S = s;
    *w = dup_vec(hw);
    *nw = static_cast<int>(hw.size());
    *off = dup_vec(ho);
    *rows = dup_vec(hr);
    *cols = dup_vec(hc);
    return 1;
}

void ref_free(void *p) { std::free(p); }

// compute_kernel_variances (v1_0_lpa_ici_2D_fused.cpp:691-717).
void ref_variances(const float *w, int nw, const int *off, const int *rows, const int *cols, int nk, float sigma,
                   float *var) {
    std::vector<float> hw(w, w + nw), v(nk, 0.0f);
    std::vector<int> ho(off, off + nk), hr(rows, rows + nk), hc(cols, cols + nk);
    compute_kernel_variances(hw, ho, hr, hc, v, sigma);
    std::memcpy(var, v.data(), sizeof(float) * nk);
}

// create_noisy_image (v1_0_lpa_ici_2D_fused.cpp:759-776).
void ref_noise(const float *clean, float *noisy, int n, float sigma, unsigned seed) {
    std::vector<float> c(clean, clean + n);
    create_noisy_image(c.data(), noisy, n, sigma, seed);
}

// calculate_PSNR (v1_0_lpa_ici_2D_fused.cpp:778-799).
double ref_psnr(const float *a, const float *b, int n) {
    std::vector<float> x(a, a + n), y(b, b + n);
    return calculate_PSNR(x.data(), y.data(), n);
}

// The CPU engine: anisotropic_lpa_ici_cpu_fused (v1_0_lpa_ici_2D_fused.cpp:851-930) or
// anisotropic_lpa_ici_cpu_naive (v0_0_lpa_ici_2D_naive.cpp:817-929).  out is zeroed first, as the
// reference's main() does.
void ref_forward(const float *noisy, float *out, int W, int H, const float *w, int nw, const int *off,
                 const int *rows, const int *cols, int D, int S, const float *var, float gamma) {
    std::vector<float> x(noisy, noisy + static_cast<size_t>(W) * H), gw(static_cast<size_t>(W) * H, 0.0f);
    std::vector<float> hw(w, w + nw), hv(var, var + D * S);
    std::vector<int> ho(off, off + D * S), hr(rows, rows + D * S), hc(cols, cols + D * S);
    std::memset(out, 0, sizeof(float) * static_cast<size_t>(W) * H);
    REF_ENGINE(x.data(), out, W, H, 1, gw.data(), D, S, hw.data(), ho.data(), hr.data(), hc.data(), hv.data(), gamma);
}

// stbi_loadf(path, ..., 1): gray float image (gamma 2.2 for 8-bit inputs).  Free with ref_stbi_free.
float *ref_stbi_loadf(const char *path, int *W, int *H) {
    int c = 0;
    return stbi_loadf(path, W, H, &c, 1);
}

void ref_stbi_free(float *p) { stbi_image_free(p); }

// stbi_load(path, ..., 1): the 8-bit gray image before the float conversion.  Free with ref_stbi_free.
unsigned char *ref_stbi_load_u8(const char *path, int *W, int *H) {
    int c = 0;
    return stbi_load(path, W, H, &c, 1);
}

// stbi_write_hdr of a one-channel float image.
int ref_stbi_write_hdr(const char *path, int W, int H, const float *data) { return stbi_write_hdr(path, W, H, 1, data); }

// stbi_loadf(path, ..., 3): interleaved RGB float image.  Free with ref_stbi_free.
float *ref_stbi_loadf_rgb(const char *path, int *W, int *H) {
    int c = 0;
    return stbi_loadf(path, W, H, &c, 3);
}

// stbi_write_hdr of an interleaved RGB float image.
int ref_stbi_write_hdr_rgb(const char *path, int W, int H, const float *data) {
    return stbi_write_hdr(path, W, H, 3, data);
}

}  // extern "C"
