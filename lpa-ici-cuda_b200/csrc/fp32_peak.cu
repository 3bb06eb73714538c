// fp32_peak.cu -- measures the FP32 pipe's peak on the current device for the two bit-exact forms of
// "multiply, round, add, round" the LPA-ICI kernels can use: scalar FMUL + FADD, and the packed form
// fma.rn.f32x2(w, x, -0) + add.rn.f32x2 (the product as an fma with a -0 addend, so that ptxas cannot
// contract it with the add).  Built into lib/liblpaici_bench.so, used by bench.py for the roofline
// denominator; not part of the C ABI.  Scalar FFMA is measured for context.
//
// Eight chains per thread; each step multiplies a neighbouring chain's value by w and adds it to its
// own, so no product can be hoisted.  Rates are element operations per second (one FMUL or FADD of
// one float = 1; one FFMA = 2).
#include <cuda_runtime.h>

namespace {
constexpr int kChains = 8;
constexpr int kIters = 2048;

__device__ __forceinline__ float2 prod2(float2 a, float2 b, float2 nz) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(nz.x), "f"(nz.y));
    return d;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__global__ void chain_ffma(float *out, float w) {
    float acc[kChains];
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) acc[i] = fmaf(acc[(i + 1) % kChains], w, acc[i]);
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void chain_muladd(float *out, float w) {
    float acc[kChains];
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = threadIdx.x * 1e-3f + i;
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) acc[i] = __fadd_rn(acc[i], __fmul_rn(acc[(i + 1) % kChains], w));
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i];
    if (s == 1234.5f) out[threadIdx.x] = s;
}

__global__ void chain_prodadd2(float *out, float w, float neg_zero) {
    float2 acc[kChains];
    const float2 w2 = make_float2(w, w), nz = make_float2(neg_zero, neg_zero);
#pragma unroll
    for (int i = 0; i < kChains; i++) acc[i] = make_float2(threadIdx.x * 1e-3f + i, i);
    for (int it = 0; it < kIters; it++)
#pragma unroll
        for (int i = 0; i < kChains; i++) acc[i] = add2(acc[i], prod2(acc[(i + 1) % kChains], w2, nz));
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < kChains; i++) s += acc[i].x + acc[i].y;
    if (s == 1234.5f) out[threadIdx.x] = s;
}

template <typename L>
float time_ms(L launch, int reps) {
    for (int w = 0; w < 2; w++) launch();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int r = 0; r < reps; r++) launch();
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}
}  // namespace

// ops_per_s[0] = scalar FFMA (2 per FFMA), [1] = scalar FMUL + FADD, [2] = packed fma(w,x,-0) + add,
// in element operations per second.  Returns 0 or a CUDA error code.
extern "C" int lpaici_bench_fp32_peak(double *ops_per_s) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float *out = nullptr;
    cudaError_t e = cudaMalloc(&out, 4096 * sizeof(float));
    if (e != cudaSuccess) return static_cast<int>(e);
    const int grid = sms * 8, block = 256, reps = 5;
    const double steps = static_cast<double>(grid) * block * kIters * kChains;
    float ms = time_ms([&] { chain_ffma<<<grid, block>>>(out, 1e-7f); }, reps);
    ops_per_s[0] = steps * 2.0 / (ms * 1e-3);
    ms = time_ms([&] { chain_muladd<<<grid, block>>>(out, 1e-7f); }, reps);
    ops_per_s[1] = steps * 2.0 / (ms * 1e-3);
    ms = time_ms([&] { chain_prodadd2<<<grid, block>>>(out, 1e-7f, -0.0f); }, reps);
    ops_per_s[2] = steps * 4.0 / (ms * 1e-3);
    e = cudaGetLastError();
    cudaFree(out);
    return static_cast<int>(e);
}
