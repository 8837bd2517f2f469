// ktm_synth.cu -- seeded synthetic traces on the device, the same recipe as
// ktm/synth.py (numpy): a sum over point scatterers of a Ricker wavelet at the
// double-square-root time source -> scatterer -> receiver, plus N(0, sigma)
// noise from a counter hash (splitmix64 of seed*2^48 + k*2^22 + j, two 32-bit
// halves through Box-Muller).  FP64 arithmetic, so the device traces agree
// with the numpy ones to float rounding when both use the same (float) sample
// interval; each sample sums the scatterers in order, so a run repeats bit for
// bit.  Test and benchmark input only.
#include "ktm_internal.cuh"

namespace ktm {
namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

struct SynthArgs {
    int ntr, nt, nscat, k0;
    double dt, freq, noise;
    unsigned long long seed;
    const float *midX, *midY, *offX, *offY;
    const double* scat;    // [nscat][5]: x, y, tau0, v, amplitude
    float* out;            // [ntr][nt]
};

__global__ void __launch_bounds__(256) synth_kernel(SynthArgs a)
{
    extern __shared__ float acc[];            // [nt]
    const int k = blockIdx.x;
    if (k >= a.ntr) return;
    for (int j = threadIdx.x; j < a.nt; j += blockDim.x) acc[j] = 0.0f;
    __syncthreads();
    const double mx = a.midX[k], my = a.midY[k], ox = a.offX[k], oy = a.offY[k];
    const double pf = 3.14159265358979323846 * a.freq;
    const int half = (int)ceil(1.5 / a.freq / a.dt) + 1;
    for (int s = 0; s < a.nscat; s++) {
        const double* sc = a.scat + 5 * s;
        const double x = sc[0], y = sc[1], t0 = sc[2], v = sc[3], amp = sc[4];
        const double ts = sqrt(t0 * t0 + ((mx - ox - x) * (mx - ox - x) + (my - oy - y) * (my - oy - y)) / (v * v));
        const double tr = sqrt(t0 * t0 + ((mx + ox - x) * (mx + ox - x) + (my + oy - y) * (my + oy - y)) / (v * v));
        const double t = ts + tr;
        const long long j0 = (long long)floor(t / a.dt) - half;
        for (int w = threadIdx.x; w <= 2 * half; w += blockDim.x) {
            const long long j = j0 + w;
            if (j < 0 || j >= a.nt) continue;
            const double q = pf * ((double)j * a.dt - t);
            const double e = q * q;
            acc[j] += (float)(amp * (1.0 - 2.0 * e) * exp(-e));   // one thread per sample
        }
        __syncthreads();   // scatterer by scatterer: every sample sums them in order (repeatable)
    }
    __syncthreads();
    const unsigned long long kk = (unsigned long long)(a.k0 + k);
    for (int j = threadIdx.x; j < a.nt; j += blockDim.x) {
        double v = acc[j];
        if (a.noise > 0.0) {
            const unsigned long long h = splitmix64((a.seed << 48) + kk * (1ULL << 22) + (unsigned long long)j);
            const double u1 = ((double)(h >> 32) + 0.5) * (1.0 / 4294967296.0);
            const double u2 = ((double)(h & 0xFFFFFFFFULL) + 0.5) * (1.0 / 4294967296.0);
            v += a.noise * sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979323846 * u2);
        }
        a.out[(size_t)k * a.nt + j] = (float)v;
    }
}

}  // namespace
}  // namespace ktm

extern "C" int ktmSynthesizeTraces(int traceNo, int tracePts, float sampleRate, const float* midX,
                                   const float* midY, const float* offX, const float* offY,
                                   int scatterNo, const double* scatterers, double freq,
                                   double noise, unsigned long long seed, int traceOffset,
                                   float* out, void* stream)
{
    if (traceNo < 0 || tracePts <= 0 || !(sampleRate > 0.0f) || scatterNo < 0 || !(freq > 0.0))
        return ktm::set_error(KTM_ERR_ARG, "ktmSynthesizeTraces: bad sizes");
    if (traceNo == 0) return ktm::set_ok();
    if (!midX || !midY || !offX || !offY || !out || (scatterNo > 0 && !scatterers))
        return ktm::set_error(KTM_ERR_ARG, "ktmSynthesizeTraces: NULL pointer");
    if ((size_t)tracePts * sizeof(float) > (size_t)ktm::kMaxSmemBytes)
        return ktm::set_error(KTM_ERR_LIMIT, "ktmSynthesizeTraces: tracePts too large");
    ktm::SynthArgs a;
    a.ntr = traceNo; a.nt = tracePts; a.nscat = scatterNo; a.k0 = traceOffset;
    a.dt = (double)sampleRate; a.freq = freq; a.noise = noise; a.seed = seed;
    a.midX = midX; a.midY = midY; a.offX = offX; a.offY = offY; a.scat = scatterers; a.out = out;
    const size_t smem = (size_t)tracePts * sizeof(float);
    KTM_CUDA_TRY(cudaFuncSetAttribute(ktm::synth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    ktm::synth_kernel<<<traceNo, 256, smem, static_cast<cudaStream_t>(stream)>>>(a);
    KTM_CUDA_TRY(cudaGetLastError());
    return ktm::set_ok();
}
