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
// in shared memory (padded rows, red.shared.add) while its warps sweep the image columns of
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

// One CTA of 32 warps per SM, 8 tau samples per lane: each FP32 shared reduction
// is a load / compare-and-swap loop, so more warps hide more of its latency; 8
// samples a lane keep the tau tables small enough for 64 registers.  The chunk's
// accumulators get 220 KB (up to 32 traces, the lane-parallel geometry's limit).
// On the 512 x 1001 line of 32,768 traces, prefolded / table weight, padded rows:
// 32 x 1, R = 8, a padding word per 4 samples 14.8 / 18.6 ms, per 8 samples 14.9 /
// 18.9; 16 x 2 15.6 / 19.6; 24 x 1, R = 16 (80 registers) 17.3 / 21.9.  Unpadded
// rows with the lanes' visiting order rotated against bank conflicts: 32 x 1, R = 8
// 19.9 / 23.6; R = 16 (spilling) 19.6 / 25.1; 20 x 2 19.8 / 24.5; 24 x 1, R = 16
// 21.7 / 26.0; 8 x 3 (72 KB) 23.6 / 27.7.
constexpr int kAdjWarps = 32;
constexpr int kAdjThreads = kAdjWarps * 32;
constexpr int kAdjR = 8;                 // tau samples per lane per run
constexpr int kAdjMinBlocks = 1;
constexpr int kPadShift = 2;             // one padding word per 4 samples
constexpr size_t kAdjSmemBudget = 220 * 1024;
static_assert(kAdjMinBlocks * (kAdjSmemBudget + 1024) <= 228 * 1024,
              "the CTAs must fit the SM's 228 KB of shared memory");

// Accumulator rows and the weight table hold sample j at word j + (j >> kPadShift).
// At one step of the scatter the lanes of a warp sit R = 8 tau samples apart, so
// their target samples lie about 8 u' apart (u' = d(t/dt)/dtau in samples per tau
// sample, 1 at zero offset and less with offset): without padding, multiples of 4 or 8
// words that share a few banks.  The padding word per 4 samples spreads them.  A row
// of n holds every j <= n + 1; rounded up to 4 words so that the arrays after the rows
// stay 16-byte aligned.
__host__ __device__ __forceinline__ int padded_pitch(int n) { return (n + (n >> kPadShift) + 2 + 3) & ~3; }

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
// samples run0 + R L + i of a run and visits them in increasing tau, so for one
// trace the target sample floor(u) mostly advances by 0 or 1.  The lane walks them
// keeping a running (sample, value, value of the next sample) and issues an atomic
// only when it leaves a sample: one red.shared per pair where u advances by a sample,
// fewer where it stalls (shallow, far offsets), two where it jumps by two or more or
// steps back (a steep Vrms increase at large offsets).  (Visiting the samples in a
// lane-rotated order instead, against bank conflicts on unpadded rows, made every
// lane jump once per run and took a third more time: 19.9 against 14.8 ms.)
// WT: 0 sqrt(j dt) table interpolated per pair, 1 sqrt.approx per pair,
//     2 prefolded (sqrt(j dt) per output sample at the write-out).
template <int PICK, int WT>
__global__ void __launch_bounds__(kAdjThreads, kAdjMinBlocks)
demigrate_merge_kernel(AdjArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Geometry& g = a.g;
    const int pitchP = padded_pitch(a.pitch);
    float* acc = reinterpret_cast<float*>(smem_raw);                    // [chunk][pitchP]
    float* crd = acc + (size_t)a.chunk * pitchP;                        // [4][chunk]
    float2* wtab = reinterpret_cast<float2*>(crd + 4 * a.chunk + ((4 * a.chunk) & 1));  // padded [nt+1]

    const int k0 = blockIdx.x * a.chunk;
    const int n = min(a.chunk, g.ntr - k0);
    for (int i = threadIdx.x; i < a.chunk * pitchP; i += kAdjThreads) acc[i] = 0.0f;
    for (int i = threadIdx.x; i < n; i += kAdjThreads) {
        crd[i] = a.midX[k0 + i];
        crd[a.chunk + i] = a.midY[k0 + i];
        crd[2 * a.chunk + i] = a.offX[k0 + i];
        crd[3 * a.chunk + i] = a.offY[k0 + i];
    }
    if (WT == 0) {
        for (int j = threadIdx.x; j <= g.nt; j += kAdjThreads) {
            const float w0 = sqrtf((float)j * g.dt), w1 = sqrtf((float)(j + 1) * g.dt);
            wtab[j + (j >> kPadShift)] = make_float2(w0, w1 - w0);
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
    // bits(fl) = K + i0, K = kMagicBits a multiple of 4: the padded word of sample i0 is
    // q + (q >> kPadShift) - kPad, kPad = K + (K >> kPadShift); the row bases carry -kPad
    const unsigned kPad = (unsigned)kMagicBits + ((unsigned)kMagicBits >> kPadShift);
    const unsigned accS = smem_u32(acc) - kPad * 4u;
    const unsigned wS = smem_u32(wtab) - kPad * 8u;
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
                    const int l = base + 2 * h + e;
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
                const unsigned rowS = accS + (unsigned)(c * pitchP) * 4u;
                const f2 DS = pk(ds, ds), DR = pk(dr, dr);
                unsigned qc = 0u, pc = 0u;
                float va = 0.0f, vb = 0.0f;
#pragma unroll
                for (int h = 0; h < kAdjR / 2; h++) {
                    const PairKin kk = pair_kin(DS, DR, S2[h], T2[h], umax, M2);
                    const unsigned pp0 = kk.q0 + (kk.q0 >> kPadShift), pp1 = kk.q1 + (kk.q1 >> kPadShift);
                    f2 VAL;
                    if (WT == 0) {
                        const float2 w0 = lds_f2(wS + pp0 * 8u), w1 = lds_f2(wS + pp1 * 8u);
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
                    const unsigned qs[2] = {kk.q0, kk.q1}, ps[2] = {pp0, pp1};
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const unsigned q = qs[e];
                        if (h == 0 && e == 0) {
                            qc = q; pc = ps[0]; va = ca[0]; vb = cb[0];
                            continue;
                        }
                        const bool same = q == qc;
                        const bool next = q == qc + 1u;
                        red_shared_if(!same, rowS + pc * 4u, va);
                        if (PICK == KTM_PICK_LINEAR) {
                            // sample qc + 1 is flushed here only where u jumped by two or more
                            const unsigned qn = qc + 1u;
                            red_shared_if(!same && !next, rowS + (qn + (qn >> kPadShift)) * 4u, vb);
                        }
                        va = same ? va + ca[e] : (next ? vb + ca[e] : ca[e]);
                        vb = same ? vb + cb[e] : cb[e];
                        qc = q;
                        pc = ps[e];
                    }
                }
                red_shared(rowS + pc * 4u, va);
                if (PICK == KTM_PICK_LINEAR) {
                    const unsigned qn = qc + 1u;
                    red_shared(rowS + (qn + (qn >> kPadShift)) * 4u, vb);
                }
            }
        }
    }
    asm volatile("" ::: "memory");     // the scatter wrote acc: no load below reuses older values
    __syncthreads();
    for (int i = threadIdx.x; i < n * a.pitch; i += kAdjThreads) {
        const int c = i / a.pitch, j = i % a.pitch;
        float v = (j > 0 && j < g.nt) ? acc[(size_t)c * pitchP + j + (j >> kPadShift)] : 0.0f;
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
    const int wt = weightMethod == KTM_WEIGHT_SQRT ? 1 : weightMethod == KTM_WEIGHT_PREFOLD ? 2 : 0;
    // the sqrt(j dt) table only for the table weight; the coordinates' alignment pad
    const size_t fixed = (wt == 0 ? (size_t)padded_pitch(g.nt + 1) * sizeof(float2) : 0) + 64;
    const size_t perTrace = (size_t)padded_pitch(pitch) * sizeof(float) + 4 * sizeof(float);
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
