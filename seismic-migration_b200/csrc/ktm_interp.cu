// ktm_interp.cu -- time-axis interpolation of traces by 2^N on the device,
// ktmInterpTraceBlock.m opt 2 (:134-154): the samples at t = 0, 1, ..., nt-1
// are linearly interpolated (Octave interp1, method 'linear') onto
// t' = 0, 1/2^N, ..., nt-1, which gives (nt-1) 2^N + 1 samples at dt / 2^N.
//
// Octave evaluates the piecewise-linear interpolant in double as
//     y = (y[i+1] - y[i]) * (t' - i) + y[i],   i = the interval of t'
// (the last point, t' = nt-1, in the last interval with t' - i = 1).  With
// float samples the difference, the offset t' - i (a multiple of 2^-N) and
// their product are exact in double, so one rounding of the sum -- an FMA
// here -- reproduces Octave's double result; the output is that value rounded
// to float.  HBM-bound: 4 bytes read per input sample, 4 * 2^N written.
#include "ktm_internal.cuh"

#include <algorithm>

namespace ktm {
namespace {

__global__ void __launch_bounds__(256) interp_kernel(const float* __restrict__ in, int inStride,
                                                    int nt, int levels, float* __restrict__ out,
                                                    int outStride, int nout)
{
    const int k = blockIdx.y;
    const float* x = in + (size_t)k * inStride;
    float* y = out + (size_t)k * outStride;
    const int mask = (1 << levels) - 1;
    const double step = 1.0 / (double)(1 << levels);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nout; j += gridDim.x * blockDim.x) {
        if (nt < 2) {
            y[j] = x[0];
            continue;
        }
        int i = j >> levels;
        double s = (double)(j & mask) * step;
        if (i >= nt - 1) {                 // the last point: last interval, offset 1
            i = nt - 2;
            s = 1.0;
        }
        const double y0 = (double)x[i], y1 = (double)x[i + 1];
        y[j] = (float)fma(y1 - y0, s, y0);
    }
}

}  // namespace

int interp_traces(const ktm_interp* p)
{
    if (!p) return set_error(KTM_ERR_ARG, "NULL interp");
    if (p->traceNo < 0 || p->tracePts < 0) return set_error(KTM_ERR_ARG, "negative sizes");
    if (p->levels < 0 || p->levels > 10) return set_error(KTM_ERR_ARG, "levels must be 0..10");
    if (p->traceNo == 0 || p->tracePts == 0) return KTM_OK;
    if (!p->in || !p->out) return set_error(KTM_ERR_ARG, "NULL buffer");
    const long long nout = ktmInterpLength(p->tracePts, p->levels);
    const int inStride = p->inStride > 0 ? p->inStride : p->tracePts;
    const long long outStride = p->outStride > 0 ? p->outStride : nout;
    if (inStride < p->tracePts) return set_error(KTM_ERR_ARG, "inStride < tracePts");
    if (outStride < nout) return set_error(KTM_ERR_ARG, "outStride < (tracePts - 1) * 2^levels + 1");
    if (nout > 0x7fffffffLL || outStride > 0x7fffffffLL)
        return set_error(KTM_ERR_LIMIT, "interpolated trace too long");
    cudaStream_t s = static_cast<cudaStream_t>(p->stream);
    // one grid row per trace (gridDim.y <= 65535: traces in slices of 65535)
    for (int k0 = 0; k0 < p->traceNo; k0 += 65535) {
        const int n = std::min(65535, p->traceNo - k0);
        const unsigned gx = (unsigned)std::min<long long>((nout + 255) / 256, 64);
        dim3 grid(gx, (unsigned)n);
        interp_kernel<<<grid, 256, 0, s>>>(p->in + (size_t)k0 * inStride, inStride, p->tracePts,
                                           p->levels, p->out + (size_t)k0 * outStride,
                                           (int)outStride, (int)nout);
        KTM_CUDA_TRY(cudaGetLastError());
    }
    return KTM_OK;
}

}  // namespace ktm

extern "C" {

long long ktmInterpLength(int tracePts, int levels)
{
    if (tracePts <= 0 || levels < 0 || levels > 30) return 0;
    return (long long)(tracePts - 1) * (1LL << levels) + 1;
}

int ktmInterpTraces(const ktm_interp* interp)
{
    int rc = ktm::interp_traces(interp);
    return rc ? rc : ktm::set_ok();
}

}  // extern "C"
