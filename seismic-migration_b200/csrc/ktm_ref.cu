// ktm_ref.cu -- reference-mode PSTM kernel: the arithmetic of psktmCPU.c:13-101
// on sm_100a, bit-identical to the reference run with one thread.
//
// How bit-identity is kept
//   * every float operation is an explicitly rounded intrinsic (__fadd_rn,
//     __fmul_rn, __fsqrt_rn, __fdiv_rn), so nothing is contracted into an FMA
//     and square root / division are IEEE round-to-nearest, as SSE sqrtss /
//     divss are in the gcc -O3 x86-64 build of psktmCPU.c;
//   * the operand order follows the C source (:46-49, :65-72, :78-85);
//   * each image sample is owned by one thread, which adds the traces in
//     increasing k, the order of the reference's outer loop (:56-59).
//
// Work decomposition (B200: 148 SMs, 32-wide warps)
//   CTA  = kWarps warps; warp w owns image column (blockIdx.x*kWarps + w).
//   warp = one column x a run of 32*R consecutive tau samples; lane L owns
//          tau = run0 + L + 32*r, r < R, so a warp reads a narrow, monotone
//          window of each trace (few shared-memory bank conflicts).
//   Traces are streamed in chunks of `chunk` traces through shared memory
//   (double-buffered with cp.async), so every trace sample is read from HBM
//   once per CTA and reused by the CTA's kWarps*32*R image samples.
#include "ktm_internal.cuh"

namespace ktm {
namespace {

constexpr int kWarps = 8;
// Two trace stages per CTA within this budget, so that three CTAs (24 warps)
// can be resident per SM.
constexpr int kRefSmemBudget = 72 * 1024;

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n"); }

// Stage traces [k0, k0+n) (samples [0, nt)) and their geometry into one buffer.
__device__ __forceinline__ void stage_chunk(float* buf, float4* geo, const Geometry& g, int k0,
                                            int n, const float* __restrict__ traces,
                                            const float* __restrict__ midX,
                                            const float* __restrict__ midY,
                                            const float* __restrict__ offX,
                                            const float* __restrict__ offY)
{
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int c = 0; c < n; c++) {
        const float* src = traces + (size_t)(k0 + c) * g.stride;
        float* dst = buf + c * g.nt;
        for (int s = tid; s < g.nt; s += nth) cp_async4(dst + s, src + s);
    }
    for (int c = tid; c < n; c += nth) {
        int k = k0 + c;
        geo[c] = make_float4(midX[k], midY[k], offX[k], offY[k]);
    }
}

template <int R>
__global__ void __launch_bounds__(kWarps * 32)
reference_kernel(Geometry g, const float* __restrict__ midX, const float* __restrict__ midY,
                 const float* __restrict__ offX, const float* __restrict__ offY,
                 const float* __restrict__ traces, const float* __restrict__ vel,
                 float* __restrict__ image, int accumulate, int chunk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4* geo = reinterpret_cast<float4*>(smem_raw);                 // [2][chunk]
    float* tbuf = reinterpret_cast<float*>(geo + 2 * chunk);            // [2][chunk][nt]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int col = blockIdx.x * kWarps + warp;
    const bool colValid = col < g.nx * g.ny;
    const int ci = colValid ? col / g.ny : 0, cj = colValid ? col % g.ny : 0;
    const int run0 = blockIdx.y * (32 * R);

    // psktmFunctions.c:26-30: axis values in float
    const float xx = __fadd_rn(g.x0, __fmul_rn(__int2float_rn(ci), g.dx));
    const float yy = __fadd_rn(g.y0, __fmul_rn(__int2float_rn(cj), g.dy));

    float tauS[R], slowS[R], acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        int l = run0 + lane + 32 * r;
        int lc = l < g.nz ? l : g.nz - 1;
        float zz = __fadd_rn(g.z0, __fmul_rn(__int2float_rn(lc), g.dz));
        tauS[r] = __fmul_rn(zz, zz);                                     // :47
        float v = vel[lc];
        slowS[r] = __fdiv_rn(1.0f, __fmul_rn(v, v));                     // :48
        acc[r] = 0.0f;
    }

    const int nchunks = (g.ntr + chunk - 1) / chunk;
    if (nchunks > 0) {
        int n0 = min(chunk, g.ntr);
        stage_chunk(tbuf, geo, g, 0, n0, traces, midX, midY, offX, offY);
        cp_async_commit();
    }
    for (int ch = 0; ch < nchunks; ch++) {
        const int buf = ch & 1;
        const int k0 = ch * chunk, n = min(chunk, g.ntr - k0);
        if (ch + 1 < nchunks) {
            int k1 = k0 + chunk, n1 = min(chunk, g.ntr - k1);
            stage_chunk(tbuf + (buf ^ 1) * chunk * g.nt, geo + (buf ^ 1) * chunk, g, k1, n1,
                        traces, midX, midY, offX, offY);
            cp_async_commit();
            cp_async_wait_1();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        const float* tb = tbuf + buf * chunk * g.nt;
        const float4* gb = geo + buf * chunk;
        if (colValid) {
            for (int c = 0; c < n; c++) {
                const float4 m = gb[c];   // midX, midY, offX, offY
                // :65-66 and :71-72, operand order of the C source
                float dxm = __fsub_rn(m.x, xx);
                float cs = __fsub_rn(dxm, m.z), cr = __fadd_rn(dxm, m.z);
                float tC = __fmul_rn(cs, cs), tD = __fmul_rn(cr, cr);
                float dym = __fsub_rn(m.y, yy);
                float ds = __fsub_rn(dym, m.w), dr = __fadd_rn(dym, m.w);
                float tA = __fadd_rn(tC, __fmul_rn(ds, ds));
                float tB = __fadd_rn(tD, __fmul_rn(dr, dr));
                const float* tr = tb + c * g.nt;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    // :78-80
                    float t = __fsqrt_rn(__fadd_rn(tauS[r], __fmul_rn(tA, slowS[r])));
                    t = __fadd_rn(t, __fsqrt_rn(__fadd_rn(tauS[r], __fmul_rn(tB, slowS[r]))));
                    int it = __float2int_rz(__fdiv_rn(t, g.dt));
                    // :82-85
                    if (it < g.nt && it > 0) {
                        float a = __fmul_rn(tr[it], t);
                        acc[r] = __fadd_rn(acc[r], __fmul_rn(a, __fsqrt_rn(__fdiv_rn(tauS[r], t))));
                    }
                }
            }
        }
        __syncthreads();
    }

    if (colValid) {
        float* out = image + (size_t)col * g.nz;
#pragma unroll
        for (int r = 0; r < R; r++) {
            int l = run0 + lane + 32 * r;
            if (l < g.nz) out[l] = accumulate ? __fadd_rn(out[l], acc[r]) : acc[r];
        }
    }
}

template <int R>
int launch_r(const Geometry& g, const float* midX, const float* midY, const float* offX,
             const float* offY, const float* traces, const float* vel, float* image,
             int accumulate, cudaStream_t stream)
{
    // chunk of traces per stage; two stages in shared memory
    const size_t perTrace = (size_t)g.nt * sizeof(float) + sizeof(float4);
    int chunk = (int)(kRefSmemBudget / (2 * perTrace));
    if (chunk < 1) chunk = (int)((kMaxSmemBytes - 1024) / (2 * perTrace));
    if (chunk < 1)
        return set_error(KTM_ERR_LIMIT,
                         "reference kernel: tracePts=%d exceeds the shared-memory stage "
                         "limit (%d samples)", g.nt, (int)((kMaxSmemBytes - 1024) / 8 - 4));
    chunk = chunk > 32 ? 32 : chunk;
    size_t smem = 2 * (size_t)chunk * perTrace;
    auto kern = reference_kernel<R>;
    KTM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    const long long cols = (long long)g.nx * g.ny;
    dim3 grid((unsigned)((cols + kWarps - 1) / kWarps), (unsigned)((g.nz + 32 * R - 1) / (32 * R)));
    if (grid.y > 65535)
        return set_error(KTM_ERR_LIMIT, "reference kernel: Nz=%d too large", g.nz);
    kern<<<grid, kWarps * 32, smem, stream>>>(g, midX, midY, offX, offY, traces, vel, image,
                                              accumulate, chunk);
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace

int launch_reference(const Geometry& g, const float* midX, const float* midY, const float* offX,
                     const float* offY, const float* traces, const float* vel, float* image,
                     int accumulate, int tileRun, cudaStream_t stream)
{
    if ((long long)g.nx * g.ny * g.nz == 0) return KTM_OK;
    if (g.ntr == 0) {
        if (!accumulate)
            KTM_CUDA_TRY(cudaMemsetAsync(image, 0,
                                         sizeof(float) * (size_t)g.nx * g.ny * g.nz, stream));
        return KTM_OK;
    }
    // Run length per warp.  Every image sample keeps its traces in reference
    // order, so the traces cannot be split across CTAs; parallelism comes from
    // the image alone: the largest R in {16, 8, 4, 2, 1} that still gives about
    // two waves of 24 resident warps per SM, and among those the least padding.
    int R = tileRun > 0 ? tileRun / 32 : 0;
    if (R == 0) {
        int dev = 0, sm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
        const long long cols = (long long)g.nx * g.ny;
        const long long wantWarps = 48LL * sm;
        R = 1;
        for (int r : {16, 8, 4, 2}) {
            const long long warps = cols * ((g.nz + 32 * r - 1) / (32 * r));
            if (warps >= wantWarps) { R = r; break; }
        }
        if (R >= 8) {
            int best = R, bestWaste = 1 << 30;
            for (int r : {16, 8, 4}) {
                if (r > R) continue;
                int run = 32 * r, waste = ((g.nz + run - 1) / run) * run - g.nz;
                if (waste < bestWaste) { bestWaste = waste; best = r; }
            }
            R = best;
        }
    }
    switch (R) {
        case 1: return launch_r<1>(g, midX, midY, offX, offY, traces, vel, image, accumulate, stream);
        case 2: return launch_r<2>(g, midX, midY, offX, offY, traces, vel, image, accumulate, stream);
        case 4: return launch_r<4>(g, midX, midY, offX, offY, traces, vel, image, accumulate, stream);
        case 8: return launch_r<8>(g, midX, midY, offX, offY, traces, vel, image, accumulate, stream);
        case 16: return launch_r<16>(g, midX, midY, offX, offY, traces, vel, image, accumulate, stream);
        default:
            return set_error(KTM_ERR_ARG, "reference kernel: tileRun must be 32, 64, 128, 256 or 512");
    }
}

}  // namespace ktm
