// ktm_adjoint.cu -- Kirchhoff demigration: the exact transpose of the fast
// migration operator (ktm_fast.cu) for its linear and truncating picks and
// its table / sqrt weights.  The reference has no adjoint; this operator is
// what least-squares migration (ktm_lsm.cu) and the dot-product test need.
//
// Migration (linear pick):  I[p] = |tau_p| sum_k s_k W_pk (q_k[i0] + f (q_k[i0+1] - q_k[i0]))
// Demigration:              D_k[i0]   += W_pk |tau_p| m[p] (1 - f)
//                           D_k[i0+1] += W_pk |tau_p| m[p] f          (0 < j < tracePts only)
// With the prefolded weight the migration reads q_k[j] sqrt(j dt) and W_pk = 1, so the
// demigration scatters without a weight and multiplies D_k[j] by sqrt(j dt) once per
// sample as it writes the chunk out.
// Every pair's (u, f, i0, W) comes from the same code as the migration's
// (ktm_pair.cuh), so the two operators are transposes pair by pair.
//
// Work decomposition: a CTA owns a chunk of traces, accumulates their samples
// in shared memory (red.shared.add) while its warps sweep the image columns of
// its column block, and writes the chunk out once (plain stores when one block
// covers all columns, red.global.add otherwise).  A warp covers one column x a
// run of 32*R tau samples at a time; the model samples, the tau tables and the
// velocity of the run stay in registers for all the chunk's traces.  FP32
// shared atomics run at ~7 per clock per SM on distinct addresses and serialise
// on equal ones, so each lane merges its own contributions before issuing them
// (demigrate_merge_kernel).
#include "ktm_pair.cuh"

#include <algorithm>

namespace ktm {
namespace {

using namespace dev;

// One CTA of 32 warps per SM, 8 tau samples per lane: the scatter is latency-
// bound (each FP32 shared reduction is a load / compare-and-swap loop), so more
// warps hide more of it; 8 samples a lane keep the tau tables small enough for
// 64 registers.  The chunk's accumulators get 220 KB (up to 32 traces, the
// lane-parallel geometry's limit).  On the 512 x 1001 line of 32,768 traces,
// prefolded / table weight: 32 x 1, R = 8: 19.9 / 23.6 ms; R = 16 (spilling) 19.6
// / 25.1; R = 4 23.1 / 26.2; 20 warps x two CTAs (R = 8) 19.8 / 24.5; 16 x 2 20.7 /
// 24.4; 24 x 2 (spilling) 20.6 / 26.3; 24 x 1, R = 16, 80 registers 21.7 / 26.0;
// 8 x 3 (72 KB) 23.6 / 27.7; before that two CTAs of 100 KB 33.4 ms and four CTAs
// of 64 registers 31.9 ms (table weight, R = 16).
constexpr int kAdjWarps = 32;
constexpr int kAdjThreads = kAdjWarps * 32;
constexpr int kAdjR = 8;                 // tau samples per lane per run
constexpr int kAdjMinBlocks = 1;
constexpr size_t kAdjSmemBudget = 220 * 1024;
static_assert(kAdjMinBlocks * (kAdjSmemBudget + 1024) <= 228 * 1024,
              "the CTAs must fit the SM's 228 KB of shared memory");
static_assert((kAdjR & (kAdjR - 1)) == 0, "the lane rotation takes a power-of-two run");

struct AdjArgs {
    Geometry g;
    const float *midX, *midY, *offX, *offY;
    const float* vel; int velCube;
    const float* image;      // model m [nx*ny][nz]
    float* data;             // [ntr][pitch] F32
    int pitch;
    int pick, weightMethod;
    float aperture;
    int chunk;               // traces per CTA
    int colsPerBlock;        // image columns per CTA (gridDim.y blocks)
    int atomicOut;           // 1: red.global.add into data (several column blocks)
};

// Volatile, so the scatter stays between the barriers around the sweep; no
// "memory" clobber, so the arithmetic around it still schedules freely.
__device__ __forceinline__ void red_shared(unsigned addr, float v)
{
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(addr), "f"(v));
}
// The same, issued only where `on` holds: a predicated instruction, no branch.
__device__ __forceinline__ void red_shared_if(bool on, unsigned addr, float v)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %2, 0;\n\t@p red.shared.add.f32 [%0], %1;\n\t}"
                 ::"r"(addr), "f"(v), "r"((unsigned)on));
}

// Lane-private merge of the scatter: lane L owns the R = kAdjR CONSECUTIVE tau
// samples run0 + R L + i of a run, so for one trace the target sample floor(u)
// advances monotonically (mostly by 0 or 1) along the lane's samples.  The lane
// walks them keeping a running (sample, value, value of the next sample) and
// issues an atomic only when it leaves a sample: one red.shared per pair where u
// advances by a sample, fewer where it stalls (shallow, far offsets), two only
// where it jumps.  Lane L visits its samples starting at i = L mod R (slot s holds
// sample (s + L) mod R), so at each step the 32 lanes sit R + 1 samples apart and
// spread over the banks; the one wrap per lane is an ordinary jump.
// WT: 0 sqrt(j dt) table interpolated per pair, 1 sqrt.approx per pair,
//     2 prefolded (sqrt(j dt) per output sample at the write-out).
template <int PICK, int WT>
__global__ void __launch_bounds__(kAdjThreads, kAdjMinBlocks)
demigrate_merge_kernel(AdjArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Geometry& g = a.g;
    float* acc = reinterpret_cast<float*>(smem_raw);                    // [chunk][pitch]
    float* crd = acc + (size_t)a.chunk * a.pitch;                       // [4][chunk]
    float2* wtab = reinterpret_cast<float2*>(crd + 4 * a.chunk + ((4 * a.chunk) & 1));  // [nt+1]

    const int k0 = blockIdx.x * a.chunk;
    const int n = min(a.chunk, g.ntr - k0);
    for (int i = threadIdx.x; i < a.chunk * a.pitch; i += kAdjThreads) acc[i] = 0.0f;
    for (int i = threadIdx.x; i < n; i += kAdjThreads) {
        crd[i] = a.midX[k0 + i];
        crd[a.chunk + i] = a.midY[k0 + i];
        crd[2 * a.chunk + i] = a.offX[k0 + i];
        crd[3 * a.chunk + i] = a.offY[k0 + i];
    }
    if (WT == 0) {
        for (int j = threadIdx.x; j <= g.nt; j += kAdjThreads) {
            const float w0 = sqrtf((float)j * g.dt), w1 = sqrtf((float)(j + 1) * g.dt);
            wtab[j] = make_float2(w0, w1 - w0);
        }
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncols = g.nx * g.ny;
    const int cb0 = blockIdx.y * a.colsPerBlock;
    const int cb1 = min(ncols, cb0 + a.colsPerBlock);
    const float invdt = 1.0f / g.dt;
    const float umax = (float)g.nt;
    const float ap2 = a.aperture > 0.0f ? a.aperture * a.aperture : -1.0f;
    const f2 M2 = pk(kMagic, kMagic);
    const unsigned accS = smem_u32(acc) - (unsigned)kMagicBits * 4u;
    const unsigned wS = smem_u32(wtab) - (unsigned)kMagicBits * 8u;
    const int nruns = (g.nz + 32 * kAdjR - 1) / (32 * kAdjR);

    for (int col = cb0 + warp; col < cb1; col += kAdjWarps) {
        const int ci = col / g.ny, cj = col % g.ny;
        const float cx = g.x0 + (float)ci * g.dx, cy = g.y0 + (float)cj * g.dy;
        for (int run = 0; run < nruns; run++) {
            const int base = run * 32 * kAdjR + kAdjR * lane;      // the lane's first sample
            f2 T2[kAdjR / 2], S2[kAdjR / 2], MT[kAdjR / 2];
            float t2min = 3.0e38f, smin = 3.0e38f;
            bool any = false;
#pragma unroll
            for (int h = 0; h < kAdjR / 2; h++) {
                float tv[2], sv[2], mv[2];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int l = base + ((2 * h + e + lane) & (kAdjR - 1));
                    const bool ok = l < g.nz;
                    const int lc = ok ? l : g.nz - 1;
                    const float tau = g.z0 + (float)lc * g.dz;
                    const float tq = tau * invdt;
                    const float v = a.velCube ? a.vel[(size_t)col * g.nz + lc] : a.vel[lc];
                    const float vd = v * g.dt;
                    tv[e] = tq * tq;
                    sv[e] = 1.0f / (vd * vd);
                    mv[e] = ok ? fabsf(tau) * a.image[(size_t)col * g.nz + l] : 0.0f;
                    if (ok) { t2min = fminf(t2min, tv[e]); smin = fminf(smin, sv[e]); }
                    any |= (mv[e] != 0.0f);
                }
                T2[h] = pk(tv[0], tv[1]);
                S2[h] = pk(sv[0], sv[1]);
                MT[h] = pk(mv[0], mv[1]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                t2min = fminf(t2min, __shfl_xor_sync(0xffffffffu, t2min, o));
                smin = fminf(smin, __shfl_xor_sync(0xffffffffu, smin, o));
            }
            if (!__any_sync(0xffffffffu, any)) continue;        // zero model in this run
            // lane c evaluates trace c's geometry for this column and run (chunk <= 32):
            // squared source / receiver distances and the keep flag (aperture, and a
            // lower bound of u over the run below the trace end); the warp then walks
            // the kept traces in increasing c, taking their distances by shuffle
            float lds_ = 0.0f, ldr_ = 0.0f;
            bool keep = false;
            if (lane < n) {
                const float mx = crd[lane], my = crd[a.chunk + lane], ox = crd[2 * a.chunk + lane],
                            oy = crd[3 * a.chunk + lane];
                const float dmx = mx - cx, dmy = my - cy;
                keep = !(ap2 >= 0.0f && dmx * dmx + dmy * dmy > ap2);
                const float sx = dmx - ox, sy = dmy - oy, rx = dmx + ox, ry = dmy + oy;
                lds_ = sx * sx + sy * sy;
                ldr_ = rx * rx + ry * ry;
                if (keep) {
                    const float ulb = sqrt_approx(fmaf(lds_, smin, t2min)) +
                                      sqrt_approx(fmaf(ldr_, smin, t2min));
                    keep = ulb < umax * 1.0001f + 1.0f;          // not past the trace end
                }
            }
            for (unsigned kept = __ballot_sync(0xffffffffu, keep); kept; kept &= kept - 1u) {
                const int c = __ffs(kept) - 1;
                const float ds = __shfl_sync(0xffffffffu, lds_, c);
                const float dr = __shfl_sync(0xffffffffu, ldr_, c);
                const unsigned rowS = accS + (unsigned)(c * a.pitch) * 4u;
                const f2 DS = pk(ds, ds), DR = pk(dr, dr);
                unsigned qc = 0u;
                float va = 0.0f, vb = 0.0f;
#pragma unroll
                for (int h = 0; h < kAdjR / 2; h++) {
                    const PairKin kk = pair_kin(DS, DR, S2[h], T2[h], umax, M2);
                    f2 VAL;
                    if (WT == 0) {
                        const float2 w0 = lds_f2(wS + kk.q0 * 8u), w1 = lds_f2(wS + kk.q1 * 8u);
                        VAL = mul2(fma2(kk.F, pk(w0.y, w1.y), pk(w0.x, w1.x)), MT[h]);
                    } else if (WT == 1) {
                        VAL = mul2(mul2(pk(sqrt_approx(kk.u0), sqrt_approx(kk.u1)),
                                        pk(sqrtf(g.dt), sqrtf(g.dt))),
                                   MT[h]);
                    } else {
                        VAL = MT[h];
                    }
                    float ca[2], cb[2];
                    if (PICK == KTM_PICK_LINEAR) {
                        const f2 B = mul2(VAL, kk.F);          // f * val       -> sample i0 + 1
                        const f2 A = sub2(VAL, B);             // (1 - f) * val -> sample i0
                        upk(A, ca[0], ca[1]);
                        upk(B, cb[0], cb[1]);
                    } else {
                        upk(VAL, ca[0], ca[1]);
                        cb[0] = cb[1] = 0.0f;
                    }
                    const unsigned qs[2] = {rowS + kk.q0 * 4u, rowS + kk.q1 * 4u};
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const unsigned q = qs[e];
                        if (h == 0 && e == 0) {
                            qc = q; va = ca[0]; vb = cb[0];
                            continue;
                        }
                        const bool same = q == qc;
                        const bool next = q == qc + 4u;
                        red_shared_if(!same, qc, va);
                        if (PICK == KTM_PICK_LINEAR) red_shared_if(!same && !next, qc + 4u, vb);
                        va = same ? va + ca[e] : (next ? vb + ca[e] : ca[e]);
                        vb = same ? vb + cb[e] : cb[e];
                        qc = q;
                    }
                }
                red_shared(qc, va);
                if (PICK == KTM_PICK_LINEAR) red_shared(qc + 4u, vb);
            }
        }
    }
    asm volatile("" ::: "memory");     // the scatter wrote acc: no load below reuses older values
    __syncthreads();
    for (int i = threadIdx.x; i < n * a.pitch; i += kAdjThreads) {
        const int c = i / a.pitch, j = i % a.pitch;
        float v = (j > 0 && j < g.nt) ? acc[i] : 0.0f;
        if (WT == 2) v *= sqrtf((float)j * g.dt);        // the fold's factor (ktm_prep.cu, ktm_lsm.cu)
        float* dst = a.data + (size_t)(k0 + c) * a.pitch + j;
        if (a.atomicOut) {
            if (v != 0.0f) atomicAdd(dst, v);
        } else {
            *dst += v;
        }
    }
}

}  // namespace

int launch_demigrate(const Geometry& g, const float* midX, const float* midY, const float* offX,
                     const float* offY, const float* vel, int velCube, const float* image,
                     float* data, int pitch, int pick, int weightMethod, float aperture,
                     int accumulate, cudaStream_t s)
{
    if (pitch < g.nt + 2 || pitch % 4 != 0)
        return set_error(KTM_ERR_ARG, "demigrate: dataPitch must be >= tracePts + 2 and a multiple of 4");
    const size_t pitchBytes = (size_t)pitch * sizeof(float);
    if (!accumulate && g.ntr > 0)
        KTM_CUDA_TRY(cudaMemsetAsync(data, 0, pitchBytes * g.ntr, s));
    if (g.ntr == 0 || (long long)g.nx * g.ny * g.nz == 0) return KTM_OK;
    const size_t fixed = (size_t)(g.nt + 1) * sizeof(float2) + 64;
    const size_t perTrace = pitchBytes + 4 * sizeof(float);
    int chunk = 32;                     // at most 32: lane c evaluates trace c's geometry
    while (chunk > 1 && fixed + chunk * perTrace > kAdjSmemBudget) chunk--;
    if (fixed + chunk * perTrace > (size_t)kMaxSmemBytes)
        return set_error(KTM_ERR_LIMIT, "demigrate: tracePts=%d exceeds the shared-memory limit", g.nt);
    const size_t smem = fixed + chunk * perTrace;

    int dev = 0, sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    const int ncols = g.nx * g.ny;
    const int chunks = (g.ntr + chunk - 1) / chunk;
    // column blocks only when the traces alone give too few CTAs (then the
    // chunks are added into the data with global atomics)
    int blocks = 1;
    const int want = 6 * sm;
    if (chunks < want) blocks = std::min((want + chunks - 1) / chunks, std::max(1, ncols / 16));
    const int perBlock = (ncols + blocks - 1) / blocks;
    blocks = (ncols + perBlock - 1) / perBlock;

    AdjArgs a;
    a.g = g; a.midX = midX; a.midY = midY; a.offX = offX; a.offY = offY;
    a.vel = vel; a.velCube = velCube; a.image = image; a.data = data; a.pitch = pitch;
    a.pick = pick; a.weightMethod = weightMethod; a.aperture = aperture;
    a.chunk = chunk; a.colsPerBlock = perBlock; a.atomicOut = blocks > 1;
    dim3 grid((unsigned)chunks, (unsigned)blocks);
#define KTM_ADJ_LAUNCH(P, W)                                                                    \
    do {                                                                                        \
        KTM_CUDA_TRY(cudaFuncSetAttribute(demigrate_merge_kernel<P, W>,                        \
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
        demigrate_merge_kernel<P, W><<<grid, kAdjThreads, smem, s>>>(a);                       \
    } while (0)
    const int wt = weightMethod == KTM_WEIGHT_SQRT ? 1 : weightMethod == KTM_WEIGHT_PREFOLD ? 2 : 0;
    if (wt == 2 && pick != KTM_PICK_LINEAR)
        return set_error(KTM_ERR_ARG, "demigrate: the prefolded weight takes the linear pick");
    if (pick == KTM_PICK_LINEAR) {
        if (wt == 2) KTM_ADJ_LAUNCH(KTM_PICK_LINEAR, 2);
        else if (wt) KTM_ADJ_LAUNCH(KTM_PICK_LINEAR, 1);
        else KTM_ADJ_LAUNCH(KTM_PICK_LINEAR, 0);
    } else {
        if (wt) KTM_ADJ_LAUNCH(KTM_PICK_TRUNCATE, 1); else KTM_ADJ_LAUNCH(KTM_PICK_TRUNCATE, 0);
    }
#undef KTM_ADJ_LAUNCH
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace ktm
