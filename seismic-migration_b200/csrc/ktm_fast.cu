// ktm_fast.cu -- the fast PSTM gather kernel (mixed precision) and the FP64
// device reference.
//
// Method (same as psktmCPU.c:56-86, extended as the north star asks):
//   image[x,tau] = |tau| * sum_k  w_k(t) * pick(trace_k, t/dt)
//   t = sqrt(tau^2 + |s-x|^2 S) + sqrt(tau^2 + |r-x|^2 S),  S = 1/v(x,tau)^2
//   w = sqrt(t)  (the reference weight t*sqrt(tau^2/t) = |tau| sqrt(t), :85)
//   pick = linear interpolation (or truncation, :80), samples outside
//   0 < j < tracePts read as zero (:82); pairs with |mid - x| > aperture skipped.
//
// Arithmetic per (image sample, trace) pair, everything in FP32:
//   a_s = T2' + Ds*S', a_r = T2' + Dr*S'   (T2' = (tau/dt)^2, S' = S/dt^2:
//                                           the traveltime comes out in samples)
//   u   = sqrt.approx(a_s) + sqrt.approx(a_r)          2 SFU ops
//   u   = min(u, nt)   (also maps NaN to nt: reads the zero guard sample)
//   i0  = floor(u) by the round-down 1.5*2^23 add, f = u - i0
//   (d, dd) = stage[i0]  (float2: sample and forward difference)
//   acc += d + f*dd                               (prefolded weight)
//   acc += sqrt.approx(u) * (d + f*dd)            (in-kernel weight, 3rd SFU op)
// The per-trace FP32 scale (F16/BF16 storage) and, when prefolded, sqrt(j*dt)
// are multiplied into the staged samples once per CTA, not once per pair.
//
// Work decomposition: CTA = kWarps warps, warp w = one image column x a run
// of 32*R tau samples (lane L owns tau = run0 + L + 32 r), one run per CTA
// (blockIdx.y).  Per chunk of traces the CTA computes, for every (trace,
// column) pair, the squared source/receiver distances and a skip flag
// (aperture, or a lower bound on u over the run beyond the trace end), so the
// inner loop branches once per trace, warp-uniformly.
#include "ktm_internal.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ktm {
namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

__device__ __forceinline__ float sqrt_approx(float x)
{
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float load_sample(const void* p, int fmt, size_t idx)
{
    if (fmt == KTM_FMT_F32) return static_cast<const float*>(p)[idx];
    if (fmt == KTM_FMT_F16) return __half2float(static_cast<const __half*>(p)[idx]);
    return __bfloat162float(static_cast<const __nv_bfloat16*>(p)[idx]);
}

struct ColInfo {
    float x, y;       // column coordinates
    float t2min;      // min over the run of (tau/dt)^2
    float smin;       // min over the run of S' = 1/(v dt)^2
};

template <int R, int PICK, int PREFOLD>
__global__ void __launch_bounds__(kThreads, 2)
fast_kernel(FastArgs a, int chunk, int ns)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* stage = reinterpret_cast<float2*>(smem_raw);                 // [chunk][ns]
    float2* geo = stage + (size_t)chunk * ns;                            // [chunk][kWarps]
    float* wtab = reinterpret_cast<float*>(geo + chunk * kWarps);        // [ns] sqrt(j*dt)
    __shared__ ColInfo cinfo[kWarps];

    const Geometry& g = a.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncols = g.nx * g.ny;
    const int col = blockIdx.x * kWarps + warp;
    const bool colValid = col < ncols;
    const int ci = colValid ? col / g.ny : 0, cj = colValid ? col % g.ny : 0;
    const int run0 = blockIdx.y * (32 * R);
    const float invdt = 1.0f / g.dt;

    // ---- per-thread tau tables -------------------------------------------
    float T2[R], S[R], acc[R];
    float t2min = 3.0e38f, smin = 3.0e38f;
    int nvalid = 0;
#pragma unroll
    for (int r = 0; r < R; r++) {
        int l = run0 + lane + 32 * r;
        bool ok = l < g.nz;
        int lc = ok ? l : g.nz - 1;
        float tau = g.z0 + (float)lc * g.dz;
        float tq = tau * invdt;
        T2[r] = tq * tq;
        float v = a.velCube ? a.vel[(size_t)(colValid ? col : 0) * g.nz + lc] : a.vel[lc];
        float vd = v * g.dt;
        S[r] = 1.0f / (vd * vd);
        acc[r] = 0.0f;
        if (ok) { t2min = fminf(t2min, T2[r]); smin = fminf(smin, S[r]); nvalid++; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t2min = fminf(t2min, __shfl_xor_sync(0xffffffffu, t2min, o));
        smin = fminf(smin, __shfl_xor_sync(0xffffffffu, smin, o));
        nvalid += __shfl_xor_sync(0xffffffffu, nvalid, o);
    }
    if (lane == 0) {
        cinfo[warp].x = g.x0 + (float)ci * g.dx;
        cinfo[warp].y = g.y0 + (float)cj * g.dy;
        cinfo[warp].t2min = t2min;
        cinfo[warp].smin = colValid ? smin : -1.0f;    // -1: column outside the image
    }
    if (PREFOLD && a.weightMode == 1) {
        for (int j = threadIdx.x; j < ns; j += kThreads) wtab[j] = sqrtf((float)j * g.dt);
    }
    __syncthreads();

    const float umax = (float)g.nt;
    const float ap2 = a.aperture > 0.0f ? a.aperture * a.aperture : -1.0f;
    unsigned long long evaluated = 0;

    const int nchunks = (g.ntr + chunk - 1) / chunk;
    for (int ch = 0; ch < nchunks; ch++) {
        const int k0 = ch * chunk, n = min(chunk, g.ntr - k0);
        // ---- stage samples: (d_j, d_{j+1} - d_j), j = 0..nt, zero guards --
        for (int c = 0; c < n; c++) {
            const size_t base = (size_t)(k0 + c) * g.stride;
            const float sc = a.scale ? a.scale[k0 + c] : 1.0f;
            float2* dst = stage + (size_t)c * ns;
            for (int j = threadIdx.x; j < ns; j += kThreads) {
                float d0 = 0.0f, d1 = 0.0f;
                if (j > 0 && j < g.nt) d0 = load_sample(a.traces, a.fmt, base + j) * sc;
                if (j + 1 < g.nt) d1 = load_sample(a.traces, a.fmt, base + j + 1) * sc;
                if (PREFOLD && a.weightMode == 1) {
                    d0 *= (j > 0 && j < g.nt) ? wtab[j] : 0.0f;
                    d1 *= (j + 1 < g.nt) ? wtab[j + 1] : 0.0f;
                }
                dst[j] = make_float2(d0, d1 - d0);
            }
        }
        // ---- per (trace, column) distances and skip flags ------------------
        for (int p = threadIdx.x; p < chunk * kWarps; p += kThreads) {
            const int c = p / kWarps, w = p % kWarps;
            float2 gd = make_float2(-1.0f, 0.0f);
            const ColInfo ciw = cinfo[w];
            if (c < n && ciw.smin >= 0.0f) {
                const int k = k0 + c;
                const float mx = a.midX[k], my = a.midY[k], ox = a.offX[k], oy = a.offY[k];
                const float dmx = mx - ciw.x, dmy = my - ciw.y;
                const float sx = dmx - ox, sy = dmy - oy, rx = dmx + ox, ry = dmy + oy;
                const float ds = sx * sx + sy * sy, dr = rx * rx + ry * ry;
                bool keep = !(ap2 >= 0.0f && dmx * dmx + dmy * dmy > ap2);
                if (keep) {
                    // lower bound of u over the run; beyond the last sample -> no contribution
                    float ulb = sqrtf(fmaf(ds, ciw.smin, ciw.t2min)) +
                                sqrtf(fmaf(dr, ciw.smin, ciw.t2min));
                    keep = ulb < umax * 1.0001f + 1.0f;
                }
                if (keep) gd = make_float2(ds, dr);
            }
            geo[p] = gd;
        }
        __syncthreads();

        if (colValid) {
            const float2* gw = geo + warp;
            for (int c = 0; c < n; c++) {
                const float2 gd = gw[c * kWarps];
                if (gd.x < 0.0f) continue;                 // warp-uniform
                evaluated += nvalid;
                const float2* tr = stage + (size_t)c * ns;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    float as = fmaf(gd.x, S[r], T2[r]);
                    float ar = fmaf(gd.y, S[r], T2[r]);
                    float u = sqrt_approx(as) + sqrt_approx(ar);
                    u = fminf(u, umax);
                    float fl = __fadd_rd(u, kMagic);
                    int i0 = __float_as_int(fl) - kMagicBits;
                    float2 dd = tr[i0];
                    if (PICK == KTM_PICK_LINEAR) {
                        float f = u - (fl - kMagic);
                        float v = fmaf(f, dd.y, dd.x);
                        if (PREFOLD) acc[r] += v;
                        else acc[r] = fmaf(sqrt_approx(u), v, acc[r]);
                    } else {
                        if (PREFOLD) acc[r] += dd.x;
                        else acc[r] = fmaf(sqrt_approx(u), dd.x, acc[r]);
                    }
                }
            }
        }
        __syncthreads();
    }

    if (colValid) {
        // weight factor |tau| (and sqrt(dt): in-kernel weight used u = t/dt)
        const float wscale = PREFOLD ? 1.0f : sqrtf(g.dt);
        float* out = a.image + (size_t)col * g.nz;
#pragma unroll
        for (int r = 0; r < R; r++) {
            int l = run0 + lane + 32 * r;
            if (l < g.nz) {
                float tau = fabsf(g.z0 + (float)l * g.dz);
                float v = acc[r] * (tau * wscale);
                out[l] = a.accumulate ? out[l] + v : v;
            }
        }
    }
    if (a.pairsEvaluated) {
        // every lane of a warp counted the same pairs; lane 0 reports the warp's
        if (lane == 0 && evaluated) atomicAdd(a.pairsEvaluated, evaluated);
    }
}

template <int R, int PICK, int PREFOLD>
int launch_t(const FastArgs& a, cudaStream_t stream)
{
    const Geometry& g = a.g;
    const int ns = g.nt + 1;
    const size_t perTrace = (size_t)ns * sizeof(float2) + kWarps * sizeof(float2);
    const size_t fixed = (size_t)ns * sizeof(float) + 64;
    // two CTAs per SM: about 113 KB each
    const size_t budget = 112 * 1024;
    int chunk = budget > fixed ? (int)((budget - fixed) / perTrace) : 0;
    if (chunk < 1) chunk = (int)((kMaxSmemBytes - fixed) / perTrace);
    if (chunk < 1)
        return set_error(KTM_ERR_LIMIT,
                         "fast kernel: tracePts=%d exceeds the shared-memory stage limit", g.nt);
    if (chunk > 32) chunk = 32;
    const size_t smem = fixed + (size_t)chunk * perTrace;
    auto kern = fast_kernel<R, PICK, PREFOLD>;
    KTM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    const long long cols = (long long)g.nx * g.ny;
    dim3 grid((unsigned)((cols + kWarps - 1) / kWarps), (unsigned)((g.nz + 32 * R - 1) / (32 * R)));
    kern<<<grid, kThreads, smem, stream>>>(a, chunk, ns);
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

template <int R>
int launch_pick(const FastArgs& a, cudaStream_t stream)
{
    if (a.pick == KTM_PICK_LINEAR)
        return a.weightMode ? launch_t<R, KTM_PICK_LINEAR, 1>(a, stream)
                            : launch_t<R, KTM_PICK_LINEAR, 0>(a, stream);
    return a.weightMode ? launch_t<R, KTM_PICK_TRUNCATE, 1>(a, stream)
                        : launch_t<R, KTM_PICK_TRUNCATE, 0>(a, stream);
}

// ---------------------------------------------------------------------------
// FP64 device reference: one thread per image sample, traces straight from
// global memory.  Slow; used to measure the error of the fast path on
// configurations too large for the CPU oracle.
// ---------------------------------------------------------------------------
__global__ void f64_kernel(FastArgs a, const int* __restrict__ cols, int ncols,
                           double* __restrict__ out)
{
    const Geometry& g = a.g;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)ncols * g.nz) return;
    const int q = (int)(idx / g.nz), l = (int)(idx % g.nz);
    const int col = cols ? cols[q] : q;
    if (col < 0 || col >= g.nx * g.ny) {      // column outside the image: NaN, no reads
        out[(size_t)q * g.nz + l] = __longlong_as_double(0x7ff8000000000000LL);
        return;
    }
    const int ci = col / g.ny, cj = col % g.ny;
    const double x = (double)g.x0 + (double)ci * (double)g.dx;
    const double y = (double)g.y0 + (double)cj * (double)g.dy;
    const double tau = (double)g.z0 + (double)l * (double)g.dz;
    const double v = a.velCube ? (double)a.vel[(size_t)col * g.nz + l] : (double)a.vel[l];
    const double S = 1.0 / (v * v), tau2 = tau * tau, dt = (double)g.dt;
    const double ap2 = a.aperture > 0.0f ? (double)a.aperture * (double)a.aperture : -1.0;
    double acc = 0.0;
    for (int k = 0; k < g.ntr; k++) {
        const double mx = a.midX[k], my = a.midY[k], ox = a.offX[k], oy = a.offY[k];
        const double dmx = mx - x, dmy = my - y;
        if (ap2 >= 0.0 && dmx * dmx + dmy * dmy > ap2) continue;
        const double sx = dmx - ox, sy = dmy - oy, rx = dmx + ox, ry = dmy + oy;
        const double t = sqrt(tau2 + (sx * sx + sy * sy) * S) + sqrt(tau2 + (rx * rx + ry * ry) * S);
        const double u = t / dt;
        if (!(u < (double)g.nt)) continue;
        const double sc = a.scale ? (double)a.scale[k] : 1.0;
        const size_t base = (size_t)k * g.stride;
        double val;
        if (a.pick == KTM_PICK_LINEAR) {
            const double fl = floor(u);
            const int i0 = (int)fl;
            const double f = u - fl;
            double d0 = (i0 > 0 && i0 < g.nt) ? (double)load_sample(a.traces, a.fmt, base + i0) : 0.0;
            double d1 = (i0 + 1 > 0 && i0 + 1 < g.nt) ? (double)load_sample(a.traces, a.fmt, base + i0 + 1) : 0.0;
            if (a.weightMode == 1) {
                d0 *= sqrt((double)i0 * dt);
                d1 *= sqrt((double)(i0 + 1) * dt);
            }
            val = (1.0 - f) * d0 + f * d1;
        } else {
            const int it = (int)u;
            val = (it > 0 && it < g.nt) ? (double)load_sample(a.traces, a.fmt, base + it) : 0.0;
            if (a.weightMode == 1) val *= sqrt((double)it * dt);
        }
        const double w = a.weightMode ? fabs(tau) : (t > 0.0 ? t * sqrt(tau2 / t) : 0.0);
        acc += w * sc * val;
    }
    out[(size_t)q * g.nz + l] = acc;
}

}  // namespace

int launch_fast(const FastArgs& a, cudaStream_t stream)
{
    const Geometry& g = a.g;
    if ((long long)g.nx * g.ny * g.nz == 0) return KTM_OK;
    if (g.nt >= (1 << 22))
        return set_error(KTM_ERR_LIMIT, "fast kernel: tracePts must be < 4194304");
    if (g.ntr == 0) {
        if (!a.accumulate)
            KTM_CUDA_TRY(cudaMemsetAsync(a.image, 0, sizeof(float) * (size_t)g.nx * g.ny * g.nz,
                                         stream));
        return KTM_OK;
    }
    int R = a.tileRun > 0 ? a.tileRun / 32 : 0;
    if (R == 0) {
        int best = 16, bestWaste = 1 << 30;
        for (int r : {16, 12, 8}) {
            int run = 32 * r, waste = ((g.nz + run - 1) / run) * run - g.nz;
            if (waste < bestWaste) { bestWaste = waste; best = r; }
        }
        R = best;
    }
    switch (R) {
        case 8: return launch_pick<8>(a, stream);
        case 12: return launch_pick<12>(a, stream);
        case 16: return launch_pick<16>(a, stream);
        default: return set_error(KTM_ERR_ARG, "fast kernel: tileRun must be 256, 384 or 512");
    }
}

int launch_f64_columns(const FastArgs& a, const int* cols, int ncols, double* out,
                       cudaStream_t stream)
{
    const long long n = (long long)ncols * a.g.nz;
    if (n == 0) return KTM_OK;
    const int th = 128;
    f64_kernel<<<(unsigned)((n + th - 1) / th), th, 0, stream>>>(a, cols, ncols, out);
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace ktm
