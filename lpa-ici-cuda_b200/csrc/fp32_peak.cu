// fp32_peak.cu -- measures the FP32 pipe's peak on the current device, the roofline denominator of
// the LPA-ICI kernels (which are FP32-issue bound: one multiply and one separately rounded add per
// tap).  Built into lib/liblpaici_bench.so, used by bench.py only; not part of the C ABI.
//
// Each thread runs CH independent chains; every chain step is one instruction per lane (scalar
// FFMA, or FMUL + FADD) or one packed f32x2 instruction (two lanes' worth).  Reported as lane
// operations per second (an FFMA lane-op is 2 FLOP, an FMUL or FADD lane-op 1 FLOP).
#include <cuda_runtime.h>

namespace {
constexpr int kChains = 8;
constexpr int kIters = 2048;

__global__ void chain_ffma(float *out, float a, float b) {
    float acc[kChains];
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) acc[i] = fmaf(acc[i], a, b);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void chain_muladd(float *out, float a, float b) {
    float acc[kChains], x[kChains];
#pragma unroll
    for (int i = 0; i < kChains; i++) {
        acc[i] = threadIdx.x * 1e-3f + i;
        x[i] = 0.5f * i + threadIdx.x;
    }
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) {
            acc[i] = __fadd_rn(acc[i], __fmul_rn(x[i], a));
            x[i] = __fadd_rn(x[i], b);
        }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i] + x[i];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void chain_muladd2(float *out, float a, float b) {
    float2 acc[kChains], x[kChains];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int i = 0; i < kChains; i++) {
        acc[i] = make_float2(threadIdx.x * 1e-3f + i, i);
        x[i] = make_float2(0.5f * i + threadIdx.x, i);
    }
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) {
            acc[i] = __fadd2_rn(acc[i], __fmul2_rn(x[i], a2));
            x[i] = __fadd2_rn(x[i], b2);
        }
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i].x + acc[i].y + x[i].x + x[i].y;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

template <typename K>
float time_kernel(K kern, int grid, int block, float *out, int reps) {
    for (int w = 0; w < 2; w++) kern<<<grid, block>>>(out, 1.0001f, 1e-7f);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int r = 0; r < reps; r++) kern<<<grid, block>>>(out, 1.0001f, 1e-7f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}
}  // namespace

// lane_ops_per_s[0] = FFMA, [1] = FMUL+FADD (scalar), [2] = FMUL2+FADD2 (packed, counted per lane
// element), each in lane operations per second.  Returns 0 or a CUDA error code.
extern "C" int lpaici_bench_fp32_peak(double *lane_ops_per_s) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float *out = nullptr;
    cudaError_t e = cudaMalloc(&out, 4096 * sizeof(float));
    if (e != cudaSuccess) return static_cast<int>(e);
    const int grid = sms * 8, block = 256, reps = 5;
    const double threads = static_cast<double>(grid) * block;
    float ms = time_kernel(chain_ffma, grid, block, out, reps);
    lane_ops_per_s[0] = threads * kIters * kChains / (ms * 1e-3);
    ms = time_kernel(chain_muladd, grid, block, out, reps);
    lane_ops_per_s[1] = threads * kIters * kChains * 3.0 / (ms * 1e-3);
    ms = time_kernel(chain_muladd2, grid, block, out, reps);
    lane_ops_per_s[2] = threads * kIters * kChains * 6.0 / (ms * 1e-3);
    e = cudaGetLastError();
    cudaFree(out);
    return static_cast<int>(e);
}
