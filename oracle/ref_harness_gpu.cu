// ref_harness_gpu.cu -- builds the reference's fastest GPU source in-process.  TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile compiles this file with REF_SOURCE = the path of
// src/v4_1_lpa_ici_2D_sparse_shared.cu of titocapovilla/lpa-ici-cuda, renaming its main(), so that
// its run-length packer (build_sparse_kernels, :826-877) can be compared with this project's packer
// on the CPU, and its GPU engine (anisotropic_lpa_ici_gpu_fused, :1122-1244) can be timed beside
// this project's kernels.  Output goes to oracle/_ref/ only; nothing of the reference is copied.
#define main lpaici_reference_main
#include REF_SOURCE
#undef main

#include <cstdlib>
#include <cstring>

extern "C" {

// build_sparse_kernels: fills caller arrays sized like the oracle's packer; returns the run count.
int ref_pack_runs(const float *w, const int *off, const int *rows, const int *cols, int nk, float *weights,
                  int *run_row, int *run_col, int *run_len, int *k_first_run, int *k_num_runs, int *k_first_weight,
                  int *n_weights) {
    std::vector<float> wt;
    std::vector<int> rr, rc, rl, kfr, knr, kfw;
    build_sparse_kernels(w, off, rows, cols, nk, wt, rr, rc, rl, kfr, knr, kfw);
    std::memcpy(weights, wt.data(), sizeof(float) * wt.size());
    std::memcpy(run_row, rr.data(), sizeof(int) * rr.size());
    std::memcpy(run_col, rc.data(), sizeof(int) * rc.size());
    std::memcpy(run_len, rl.data(), sizeof(int) * rl.size());
    std::memcpy(k_first_run, kfr.data(), sizeof(int) * nk);
    std::memcpy(k_num_runs, knr.data(), sizeof(int) * nk);
    std::memcpy(k_first_weight, kfw.data(), sizeof(int) * nk);
    *n_weights = static_cast<int>(wt.size());
    return static_cast<int>(rr.size());
}

// anisotropic_lpa_ici_gpu_fused with host buffers, as the reference's main() calls it.
void ref_gpu_fused(const float *noisy, float *out, int W, int H, const float *w, int nw, const int *off,
                   const int *rows, const int *cols, int D, int S, const float *var, float gamma) {
    std::vector<float> x(noisy, noisy + static_cast<size_t>(W) * H), gw(static_cast<size_t>(W) * H, 0.0f);
    std::vector<float> hw(w, w + nw), hv(var, var + D * S);
    std::vector<int> ho(off, off + D * S), hr(rows, rows + D * S), hc(cols, cols + D * S);
    std::memset(out, 0, sizeof(float) * static_cast<size_t>(W) * H);
    anisotropic_lpa_ici_gpu_fused(x.data(), out, W, H, 1, gw.data(), D, S, hw.data(), nw, ho.data(), hr.data(),
                                  hc.data(), hv.data(), gamma);
}

}  // extern "C"
