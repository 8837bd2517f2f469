// ktm_prep.cu -- trace preparation on the device: the rho (half-derivative)
// pre-filter of scripts/ktmApplyRhoFilter.m, the sqrt(t) weight fold, per-trace
// scaling, FP16/BF16 quantisation and packing for the fast migration kernel.
//
// One CTA prepares a PAIR of traces.  With the rho filter on, the two real
// traces x and y go through ONE complex FFT as z = x + i y: every rho filter
// is Hermitian (H(-w) = conj H(w), ktmApplyRhoFilter.m:39-58), so filtering z
// and taking real and imaginary parts gives the two filtered traces.  The
// Nyquist bin, where the script's filter is not Hermitian (2.5D), is the one
// place this needs care: real(ifft(H X)) only sees Re(H) there, so Re(H) is
// what is applied.  The FFT is an in-place radix-2 Cooley-Tukey transform in
// shared memory (M = 2^ceil(log2 tracePts) complex values, M <= 16384).
//
// Output record of trace k (ktmPrepareTraces in include/ktm.h):
//   out[k][j] = Q(x'_j / s_k), x'_j = filtered x_j (times sqrt(j dt) when
//   prefold), 0 < j < tracePts; out[k][0] = out[k][j >= tracePts] = 0.
//   s_k = max|x'| (BF16), max|x'| / 32768 (F16), 1 (F32).
#include "ktm_ibm.cuh"
#include "ktm_internal.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

namespace ktm {
namespace {

constexpr int kPrepThreads = 512;
constexpr int kMaxFft = 16384;

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) { return __brev(v) >> (32 - bits); }

// In-place forward FFT (e^{-2 pi i k n / M}) of z[M] in shared memory; tw[k] = e^{-2 pi i k/M}.
__device__ void fft_inplace(float2* z, const float2* tw, int M, int logM)
{
    for (int s = 1; s <= logM; s++) {
        const int half = 1 << (s - 1);
        const int step = M >> s;          // twiddle stride
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            const int pos = b & (half - 1);
            const int i = ((b >> (s - 1)) << s) + pos;
            const int j = i + half;
            const float2 t = cmul(tw[pos * step], z[j]);
            const float2 u = z[i];
            z[i] = make_float2(u.x + t.x, u.y + t.y);
            z[j] = make_float2(u.x - t.x, u.y - t.y);
        }
        __syncthreads();
    }
}

// H at FFT bin k (natural order), frequency index kk = k - M (k >= M/2), as
// ktmApplyRhoFilter.m:33 pairs omega = 2 pi kk / Dr with the shifted spectrum.
__device__ __forceinline__ float2 rho_response(int k, int M, double dt, int opt)
{
    const int kk = k < (M >> 1) ? k : k - M;
    const double w = 2.0 * 3.14159265358979323846 * (double)kk / dt;
    const bool nyq = (k == (M >> 1));
    if (opt == KTM_RHO_2D) return make_float2((float)fabs(w), 0.0f);
    if (opt == KTM_RHO_25D) {
        const double a = sqrt(fabs(w));
        const double c = 0.70710678118654752440;    // cos(pi/4) = sin(pi/4)
        const double sgn = kk > 0 ? 1.0 : (kk < 0 ? -1.0 : 0.0);
        if (nyq) return make_float2((float)(a * c), 0.0f);
        return make_float2((float)(a * c), (float)(a * c * sgn));
    }
    // 3D: i omega (zero real part, so zero at Nyquist)
    if (nyq) return make_float2(0.0f, 0.0f);
    return make_float2(0.0f, (float)w);
}

__device__ __forceinline__ float block_max(float v, float* red)
{
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = l < (blockDim.x >> 5) ? red[l] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (l == 0) red[32] = v;
    }
    __syncthreads();
    float r = red[32];
    __syncthreads();
    return r;
}

template <int FMT>
__device__ __forceinline__ void store_q(void* out, size_t idx, float v)
{
    if (FMT == KTM_FMT_F32) static_cast<float*>(out)[idx] = v;
    else if (FMT == KTM_FMT_F16) static_cast<__half*>(out)[idx] = __float2half_rn(v);
    else static_cast<__nv_bfloat16*>(out)[idx] = __float2bfloat16_rn(v);
}

struct PrepArgs {
    int ntr, nt, inStride, pitch;
    float dt;
    const float* in;
    int ibm;                 // 1: in holds IBM-32 words
    int rho, scriptOrder, prefold;
    void* out;
    float* scale;
    int M, logM;
};

// input sample n of the trace at p (IBM words converted as ktmIBM32toIEEE does)
__device__ __forceinline__ float load_in(const float* p, int n, int ibm)
{
    if (ibm) return dev::ibm32_to_f32(reinterpret_cast<const uint32_t*>(p)[n]);
    return p[n];
}

template <int FMT>
__global__ void __launch_bounds__(kPrepThreads) prep_kernel(PrepArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* z = reinterpret_cast<float2*>(smem_raw);                 // [M] (or [nt] samples x,y)
    float2* tw = z + a.M;                                            // [M/2] twiddles
    __shared__ float red[33];

    const int k0 = 2 * blockIdx.x;
    const bool two = k0 + 1 < a.ntr;
    const float* x = a.in + (size_t)k0 * a.inStride;
    const float* y = two ? x + a.inStride : nullptr;

    if (a.rho != KTM_RHO_NONE) {
        const int M = a.M;
        for (int k = threadIdx.x; k < (M >> 1); k += blockDim.x) {
            float s, c;
            sincospif(2.0f * (float)k / (float)M, &s, &c);
            tw[k] = make_float2(c, -s);
        }
        // bit-reversed load of z = x + i y, zero padded to M (fft(trace', M), :37)
        for (int n = threadIdx.x; n < M; n += blockDim.x) {
            float xr = n < a.nt ? load_in(x, n, a.ibm) : 0.0f;
            float yi = (two && n < a.nt) ? load_in(y, n, a.ibm) : 0.0f;
            z[bitrev((unsigned)n, a.logM)] = make_float2(xr, yi);
        }
        __syncthreads();
        fft_inplace(z, tw, M, a.logM);
        // multiply by the filter, then inverse FFT as conj(FFT(conj(.))) / M
        for (int k = threadIdx.x; k < M; k += blockDim.x) {
            float2 h = rho_response(k, M, (double)a.dt, a.rho);
            float2 v = cmul(h, z[k]);
            z[k] = make_float2(v.x, -v.y);
        }
        __syncthreads();
        // bit-reverse permutation in place (swap pairs once)
        for (int n = threadIdx.x; n < M; n += blockDim.x) {
            unsigned r = bitrev((unsigned)n, a.logM);
            if ((unsigned)n < r) {
                float2 t = z[n];
                z[n] = z[r];
                z[r] = t;
            }
        }
        __syncthreads();
        fft_inplace(z, tw, M, a.logM);
        const float invM = 1.0f / (float)M;
        // result: conj(.) / M; real part = filtered x, imag (after conj) = filtered y
        for (int n = threadIdx.x; n < a.nt; n += blockDim.x)
            z[n] = make_float2(z[n].x * invM, -z[n].y * invM);
        __syncthreads();
    } else {
        for (int n = threadIdx.x; n < a.nt; n += blockDim.x)
            z[n] = make_float2(load_in(x, n, a.ibm), two ? load_in(y, n, a.ibm) : 0.0f);
        __syncthreads();
    }

    // weight fold, sample window, absmax
    float mx = 0.0f, my = 0.0f;
    for (int n = threadIdx.x; n < a.nt; n += blockDim.x) {
        float2 v = z[n];
        if (n == 0) v = make_float2(0.0f, 0.0f);
        if (a.prefold) {
            float w = sqrtf((float)n * a.dt);
            v.x *= w;
            v.y *= w;
        }
        z[n] = v;
        mx = fmaxf(mx, fabsf(v.x));
        my = fmaxf(my, fabsf(v.y));
    }
    __syncthreads();
    mx = block_max(mx, red);
    my = block_max(my, red);
    const float target = FMT == KTM_FMT_F16 ? 32768.0f : 1.0f;
    const float sx = FMT == KTM_FMT_F32 ? 1.0f : (mx > 0.0f ? mx / target : 1.0f);
    const float sy = FMT == KTM_FMT_F32 ? 1.0f : (my > 0.0f ? my / target : 1.0f);
    const float ix = 1.0f / sx, iy = 1.0f / sy;

    // output slots (the script's rotation for odd traceNo: out[q] = in[(q+1) mod n])
    int ox = k0, oy = k0 + 1;
    if (a.scriptOrder && (a.ntr & 1) && a.ntr > 1) {
        ox = (k0 + a.ntr - 1) % a.ntr;
        oy = (k0 + a.ntr) % a.ntr;
    }
    for (int n = threadIdx.x; n < a.pitch; n += blockDim.x) {
        float2 v = n < a.nt ? z[n] : make_float2(0.0f, 0.0f);
        store_q<FMT>(a.out, (size_t)ox * a.pitch + n, v.x * ix);
        if (two) store_q<FMT>(a.out, (size_t)oy * a.pitch + n, v.y * iy);
    }
    if (threadIdx.x == 0) {
        a.scale[ox] = sx;
        if (two) a.scale[oy] = sy;
    }
}

__global__ void widen_kernel(const void* __restrict__ in, int fmt, const float* __restrict__ scale,
                             int ntr, int nt, int stride, float* __restrict__ out)
{
    const size_t n = (size_t)ntr * nt;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t k = i / nt, j = i % nt;
        const size_t src = k * stride + j;
        float v = fmt == KTM_FMT_F16 ? __half2float(static_cast<const __half*>(in)[src])
                                     : __bfloat162float(static_cast<const __nv_bfloat16*>(in)[src]);
        if (scale) v *= scale[k];
        out[i] = v;
    }
}

}  // namespace

int widen_traces(const void* in, int fmt, const float* scale, int ntr, int nt, int stride,
                 void** out, cudaStream_t s)
{
    *out = nullptr;
    const size_t n = (size_t)ntr * nt;
    if (n == 0) return KTM_OK;
    KTM_CUDA_TRY(pool_malloc(out, n * sizeof(float), s));
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 65535 * 8);
    widen_kernel<<<blocks, 256, 0, s>>>(in, fmt, scale, ntr, nt, stride, static_cast<float*>(*out));
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

int packed_pitch(int nt, int fmt)
{
    const int esize = fmt == KTM_FMT_F32 ? 4 : 2;
    const int per16 = 16 / esize;
    return ((nt + 2 + per16 - 1) / per16) * per16;
}

int prepare_traces(const ktm_prep* p)
{
    if (!p) return set_error(KTM_ERR_ARG, "NULL prep");
    if (p->traceNo < 0 || p->tracePts < 0) return set_error(KTM_ERR_ARG, "negative sizes");
    if (p->outFormat < KTM_FMT_F32 || p->outFormat > KTM_FMT_BF16)
        return set_error(KTM_ERR_ARG, "bad outFormat %d", p->outFormat);
    if (p->rho < KTM_RHO_NONE || p->rho > KTM_RHO_3D) return set_error(KTM_ERR_ARG, "bad rho %d", p->rho);
    if (p->inFormat != KTM_FMT_F32 && p->inFormat != KTM_FMT_IBM32)
        return set_error(KTM_ERR_ARG, "bad inFormat %d (F32 or IBM32)", p->inFormat);
    if (!(p->sampleRate > 0.0f)) return set_error(KTM_ERR_ARG, "sampleRate must be > 0");
    if (p->traceNo == 0) return KTM_OK;
    if (!p->in || !p->out || !p->outScale) return set_error(KTM_ERR_ARG, "NULL buffer");
    PrepArgs a;
    a.ntr = p->traceNo; a.nt = p->tracePts;
    a.inStride = p->inStride > 0 ? p->inStride : p->tracePts;
    if (a.inStride < a.nt) return set_error(KTM_ERR_ARG, "inStride < tracePts");
    a.pitch = p->outPitch > 0 ? p->outPitch : packed_pitch(p->tracePts, p->outFormat);
    const int esize = p->outFormat == KTM_FMT_F32 ? 4 : 2;
    if (a.pitch < a.nt + 2 || (a.pitch * esize) % 16 != 0)
        return set_error(KTM_ERR_ARG, "outPitch must be >= tracePts + 2 and a multiple of 16 bytes");
    if (reinterpret_cast<uintptr_t>(p->out) % 16 != 0)
        return set_error(KTM_ERR_ARG, "out must be 16-byte aligned");
    a.dt = p->sampleRate; a.in = p->in; a.ibm = p->inFormat == KTM_FMT_IBM32; a.rho = p->rho; a.scriptOrder = p->rhoScriptOrder;
    a.prefold = p->prefold; a.out = p->out; a.scale = p->outScale;
    a.M = 1; a.logM = 0;
    while (a.M < a.nt) { a.M <<= 1; a.logM++; }
    size_t smem;
    if (a.rho != KTM_RHO_NONE) {
        if (a.M > kMaxFft)
            return set_error(KTM_ERR_LIMIT, "rho filter: tracePts > %d", kMaxFft);
        smem = (size_t)a.M * sizeof(float2) + (size_t)(a.M / 2 > 0 ? a.M / 2 : 1) * sizeof(float2);
    } else {
        if ((size_t)a.nt * sizeof(float2) > (size_t)kMaxSmemBytes)
            return set_error(KTM_ERR_LIMIT, "prepare: tracePts > %d", kMaxSmemBytes / 8);
        smem = (size_t)(a.nt > 0 ? a.nt : 1) * sizeof(float2);
        a.M = a.nt;
    }
    cudaStream_t s = static_cast<cudaStream_t>(p->stream);
    const unsigned grid = (unsigned)((a.ntr + 1) / 2);
    switch (p->outFormat) {
        case KTM_FMT_F32:
            KTM_CUDA_TRY(cudaFuncSetAttribute(prep_kernel<KTM_FMT_F32>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            prep_kernel<KTM_FMT_F32><<<grid, kPrepThreads, smem, s>>>(a);
            break;
        case KTM_FMT_F16:
            KTM_CUDA_TRY(cudaFuncSetAttribute(prep_kernel<KTM_FMT_F16>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            prep_kernel<KTM_FMT_F16><<<grid, kPrepThreads, smem, s>>>(a);
            break;
        default:
            KTM_CUDA_TRY(cudaFuncSetAttribute(prep_kernel<KTM_FMT_BF16>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            prep_kernel<KTM_FMT_BF16><<<grid, kPrepThreads, smem, s>>>(a);
            break;
    }
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace ktm

extern "C" {

int ktmPackedPitch(int tracePts, int format) { return ktm::packed_pitch(tracePts, format); }

int ktmPrepareTraces(const ktm_prep* prep)
{
    int rc = ktm::prepare_traces(prep);
    return rc ? rc : ktm::set_ok();
}

}  // extern "C"
