// ktm_probe.cu -- pipe-throughput probes that give the roofline denominators
// of the migration kernels on the GPU they run on: the special-function unit
// (sqrt.approx.f32, the two per-pair square roots) and the FP32 FMA pipe.
// Every probe runs independent dependency chains in enough warps that the
// pipe, not the latency, binds; the result is operations per second.
#include "ktm_internal.cuh"

namespace ktm {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 2048;

__global__ void __launch_bounds__(256) probe_sqrt(float* sink, float seed)
{
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = seed + threadIdx.x * 1e-3f + c;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) {
            float y;
            asm volatile("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v[c]));
            v[c] = y + 1.0f;   // stays near the fixed point of x -> sqrt(x) + 1
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += v[c];
    if (s == 12345.678f) sink[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) probe_rsqrt(float* sink, float seed)
{
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = seed + threadIdx.x * 1e-3f + c;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) {
            float y;
            asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v[c]));
            v[c] = y + 1.0f;
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += v[c];
    if (s == 12345.678f) sink[threadIdx.x] = s;
}

__global__ void __launch_bounds__(256) probe_ffma(float* sink, float seed)
{
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) v[c] = seed + threadIdx.x * 1e-3f + c;
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int c = 0; c < kChains; c++) {
            float y;
            asm volatile("fma.rn.f32 %0, %1, %2, %3;" : "=f"(y) : "f"(v[c]), "f"(0.999f), "f"(0.001f));
            v[c] = y;
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += v[c];
    if (s == 12345.678f) sink[threadIdx.x] = s;
}

template <class K>
int time_probe(K kern, int sm, double* opsPerSec)
{
    float* sink = nullptr;
    KTM_CUDA_TRY(cudaMalloc(&sink, 256 * sizeof(float)));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm * 8;   // 64 warps per SM
    kern<<<blocks, 256>>>(sink, 1.5f);            // warm-up
    cudaEventRecord(e0);
    const int reps = 5;
    for (int r = 0; r < reps; r++) kern<<<blocks, 256>>>(sink, 1.5f);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) return set_error(KTM_ERR_CUDA, "probe: %s", cudaGetErrorString(err));
    const double ops = (double)reps * blocks * 256.0 * kIters * kChains;
    *opsPerSec = ops / (ms * 1e-3);
    return KTM_OK;
}

}  // namespace
}  // namespace ktm

extern "C" int ktmProbePeaks(double* sqrtPerSec, double* rsqrtPerSec, double* ffmaPerSec)
{
    int dev = 0, sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    int rc;
    if (sqrtPerSec && (rc = ktm::time_probe(ktm::probe_sqrt, sm, sqrtPerSec))) return rc;
    if (rsqrtPerSec && (rc = ktm::time_probe(ktm::probe_rsqrt, sm, rsqrtPerSec))) return rc;
    if (ffmaPerSec && (rc = ktm::time_probe(ktm::probe_ffma, sm, ffmaPerSec))) return rc;
    return ktm::set_ok();
}
