// fp32_probe.cu -- FP32 FMA throughput of this GPU (no counterpart in the reference).  A measurement
// probe for bench.py, built into its own library (lib/libkami_fp32_probe.so), not the solver's:
//
//   extern "C" int kami_fp32_peak(int device, double* tflops_fma, double* tflops_fma2);
//
// returns 0 or the cudaError_t of the failing call, and restores the calling thread's device.
//
// The fused step is bound by FP32 instruction issue, so its roofline needs the FP32 peak, which the
// HBM / tensor measurements do not give.  Each thread runs 8 independent FMA chains (a * x + b with
// |a| < 1, so the values settle and never overflow), enough independent work per warp to keep the
// FMA pipes busy at full occupancy.  The packed form runs the same chains on float2 pairs with
// sm_100's FFMA2.  Results land in memory only behind a test that never holds, which keeps the
// chains live.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float a, float b) {
    float acc[kChains];
#pragma unroll
    for (int k = 0; k < kChains; k++) acc[k] = 1e-3f * (float)threadIdx.x + (float)k;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) acc[k] = fmaf(acc[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; k++) s += acc[k];
    if (s == -1.f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) fma2_probe_kernel(float* out, int iters, float a, float b) {
    float2 acc[kChains];
    const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
    for (int k = 0; k < kChains; k++) acc[k] = make_float2(1e-3f * (float)threadIdx.x + (float)k, (float)k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) acc[k] = __ffma2_rn(acc[k], a2, b2);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kChains; k++) s += acc[k].x + acc[k].y;
    if (s == -1.f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

cudaError_t measure_fp32_peak(int sm_count, double* tflops_fma, double* tflops_fma2) {
    const int threads = 256, blocks = sm_count * 8, iters = 1 << 15;
    float* out = nullptr;
    cudaError_t e = cudaMalloc(&out, sizeof(float) * (size_t)blocks * threads);
    if (e != cudaSuccess) return e;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if ((e = cudaEventCreate(&t0)) == cudaSuccess) e = cudaEventCreate(&t1);
    const double fmas = (double)blocks * threads * iters * kChains;
    for (int packed = 0; packed < 2 && e == cudaSuccess; packed++) {
        float best = 0.f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {  // the first launch warms up
            e = cudaEventRecord(t0, 0);
            if (packed)
                fma2_probe_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
            else
                fma_probe_kernel<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
            if (e == cudaSuccess) e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaEventRecord(t1, 0);
            if (e == cudaSuccess) e = cudaEventSynchronize(t1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
            if (e == cudaSuccess && rep > 0 && (best == 0.f || ms < best)) best = ms;
        }
        const double tf = best > 0.f ? 2.0 * fmas * (packed ? 2.0 : 1.0) / (best * 1e-3) / 1e12 : 0.0;
        *(packed ? tflops_fma2 : tflops_fma) = tf;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(out);
    return e;
}

}  // namespace

extern "C" int kami_fp32_peak(int device, double* tflops_fma, double* tflops_fma2) {
    if (!tflops_fma || !tflops_fma2) return (int)cudaErrorInvalidValue;
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return (int)e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return (int)e;
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = measure_fp32_peak(sms, tflops_fma, tflops_fma2);
    cudaSetDevice(prev);  // the caller's thread keeps its device
    return (int)e;
}
