// ktm_ibm.cu -- IBM-32 -> IEEE conversion kernel and its C entry points
// (ktmIBM32toIEEE, same name and arguments as ioFunctions.c:4, and the
// device-buffer form).  An elementwise HBM-bound pass: 4 bytes read and 4
// written per sample; 16-byte vector loads and stores where the buffers allow.
#include "ktm_ibm.cuh"
#include "ktm_internal.cuh"

#include <algorithm>

namespace ktm {
namespace {

__global__ void __launch_bounds__(256) ibm_kernel(const uint32_t* __restrict__ in,
                                                  float* __restrict__ out, size_t n, int vec)
{
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nth = (size_t)gridDim.x * blockDim.x;
    size_t head = 0;
    if (vec) {
        const size_t n4 = n / 4;
        const uint4* in4 = reinterpret_cast<const uint4*>(in);
        float4* out4 = reinterpret_cast<float4*>(out);
        for (size_t i = tid; i < n4; i += nth) {
            const uint4 w = __ldcs(in4 + i);
            float4 v;
            v.x = dev::ibm32_to_f32(w.x);
            v.y = dev::ibm32_to_f32(w.y);
            v.z = dev::ibm32_to_f32(w.z);
            v.w = dev::ibm32_to_f32(w.w);
            __stcs(out4 + i, v);
        }
        head = n4 * 4;
    }
    for (size_t i = head + tid; i < n; i += nth) out[i] = dev::ibm32_to_f32(__ldcs(in + i));
}

}  // namespace

int ibm_to_ieee(const uint32_t* in, float* out, size_t n, cudaStream_t s)
{
    if (n == 0) return KTM_OK;
    if (!in || !out) return set_error(KTM_ERR_ARG, "NULL buffer");
    int dev = 0, sms = 148;
    KTM_CUDA_TRY(cudaGetDevice(&dev));
    KTM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int vec = (reinterpret_cast<uintptr_t>(in) % 16 == 0) &&
                    (reinterpret_cast<uintptr_t>(out) % 16 == 0);
    const size_t units = vec ? (n + 3) / 4 : n;
    const size_t want = (units + 255) / 256;
    const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)sms * 8));
    ibm_kernel<<<grid, 256, 0, s>>>(in, out, n, vec);
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace ktm

extern "C" {

int ktmIBM32toIEEEDevice(const unsigned int* input, float* output, size_t n, void* stream)
{
    int rc = ktm::ibm_to_ieee(input, output, n, static_cast<cudaStream_t>(stream));
    return rc ? rc : ktm::set_ok();
}

void ktmIBM32toIEEE(unsigned int* input, float* output, int n)
{
    if (n <= 0) {
        ktm::set_ok();
        return;
    }
    if (!input || !output) {
        ktm::set_error(KTM_ERR_ARG, "NULL buffer");
        return;
    }
    const size_t bytes = (size_t)n * 4;
    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, 2 * bytes);
    if (e != cudaSuccess) {
        ktm::set_error(e == cudaErrorMemoryAllocation ? KTM_ERR_NOMEM : KTM_ERR_CUDA,
                       "ktmIBM32toIEEE: %s", cudaGetErrorString(e));
        return;
    }
    uint32_t* din = static_cast<uint32_t*>(d);
    float* dout = reinterpret_cast<float*>(din + n);
    int rc = KTM_OK;
    e = cudaMemcpy(din, input, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        rc = ktm::ibm_to_ieee(din, dout, (size_t)n, nullptr);
        if (!rc) e = cudaMemcpy(output, dout, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    if (rc) return;
    if (e != cudaSuccess) {
        ktm::set_error(KTM_ERR_CUDA, "ktmIBM32toIEEE: %s", cudaGetErrorString(e));
        return;
    }
    ktm::set_ok();
}

}  // extern "C"
