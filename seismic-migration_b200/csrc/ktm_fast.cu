// ktm_fast.cu -- the fast PSTM gather kernel (mixed precision) and the FP64
// device reference.
//
// Method (psktmCPU.c:56-86, extended with linear pick, aperture, a Vrms cube and
// packed FP16 / BF16 / FP32 samples with a per-trace scale):
//   image[x,tau] = |tau| * sum_k  s_k * w(t) * pick(q_k, t/dt)
//   t = sqrt(tau^2 + |s-x|^2 S) + sqrt(tau^2 + |r-x|^2 S),  S = 1/v(x,tau)^2
//   reference weight t*sqrt(tau^2/t) = |tau| sqrt(t) (:85): |tau| per image
//   sample, sqrt(t) per pair (truncating pick) or folded into the samples as
//   sqrt(j dt) by ktmPrepareTraces (linear pick);
//   pick: linear interpolation, or truncation (:80); samples outside
//   0 < j < tracePts are zero guards of the packed layout (:82);
//   pairs with |mid - x| > aperture are skipped.
//
// Input: a PACKED trace set (ktm_prep.cu): [traceNo][pitch] F32/F16/BF16 with
// zero guard samples, a per-trace FP32 scale s_k.
//
// Per (image sample, trace) pair, FP32 with two pairs per packed f32x2 op:
//   a_s = T2' + Ds*S', a_r = T2' + Dr*S'  (T2' = (tau/dt)^2, S' = S/dt^2, so
//                                          the traveltime comes out in samples)
//   u   = sqrt(a_s) + sqrt(a_r)           2 SFU ops (sqrt.approx)
//   u   = min(u, nt)   (also maps NaN to nt, a zero guard)
//   i0  = floor(u) via the round-down add of 1.5*2^23, f = u - i0
//   v   = q[i0] + f (q[i0+1] - q[i0]);  acc += s_k * v
// Work decomposition (148 SMs, 24 warps per SM at 80 registers; the CTA shape
// CtaShape below: 24 columns x one CTA per SM by default, 12 x 2 or 8 x 3):
//   warp   = one image column x a run of 32*R tau samples (lane L owns
//            tau = run0 + L + 32 r): a warp reads a narrow window of a trace;
//   CTA    = W columns (blockIdx.x) x one run (blockIdx.y) x one slice of the
//            traces (blockIdx.z); slices write partial images that a second
//            kernel sums in a fixed order (deterministic), so small images still
//            fill the GPU;
//   traces stream through shared memory in chunks, double-buffered: thread 0
//   moves a chunk's packed rows (one contiguous, 16-byte aligned range) with a
//   single bulk copy (cp.async.bulk) completed on the buffer's mbarrier, waited
//   for with a one-second bound; the coordinates and scales follow in 4-byte
//   cp.async.  For each chunk, lane c of every warp computes trace c's squared
//   distances and skip flag (aperture, or a lower bound of u over the run beyond
//   the trace end) for the warp's column; the warp walks the kept traces of its
//   ballot, taking their distances by shuffle, with no second barrier per chunk.
//   ktmAutotuneTile picks R, the shape and the chunk per job.
#include "ktm_pair.cuh"

#include <algorithm>
#include <vector>

namespace ktm {
namespace {

// CTA shapes of the fast kernels: warps per CTA (one image column each), CTAs per
// SM and dynamic shared memory per CTA.  Every shape runs 24 warps per SM with
// registers capped at 80 (65,536 / 768 threads); MB x (budget + up to 1 KB of
// static shared memory + the 1 KB the SM reserves) fits the SM's 228 KB.  More
// columns per CTA share each staged chunk of traces among more warps: on the
// 200 x 200 x 1501 image, 8192 FP16 traces, 24 x 1 takes 201.8 ms, 12 x 2 203.7
// ms and 8 x 3 208.6 ms per launch (8 x 2 225.7, 16 x 1 226.8, 4 x 6 229.6).
// Full = 1: every pick / weight / gradient path is built for the shape; 0: the
// linear pick with the prefolded or table weight only (the paths the tile
// tuner searches).
template <int W, int MB, int KB, int FULL>
struct CtaShape {
    static constexpr int kWarps = W;
    static constexpr int kThreads = W * 32;
    static constexpr int kMinBlocks = MB;
    static constexpr size_t kBudget = (size_t)KB * 1024;
    static constexpr bool kFull = FULL != 0;
};
using Shape24 = CtaShape<24, 1, 220, 1>;
using Shape12 = CtaShape<12, 2, 110, 0>;
using Shape8 = CtaShape<8, 3, 74, 0>;
template <class SH>
constexpr bool shape_fits()
{
    return SH::kMinBlocks * (SH::kBudget + 2048) <= 228 * 1024;
}
static_assert(shape_fits<Shape24>() && shape_fits<Shape12>() && shape_fits<Shape8>(),
              "each shape's CTAs must fit the SM's 228 KB of shared memory");
constexpr int kMaxChunk = 32;        // lane c of a warp evaluates trace c of a chunk
// index of the lowest set bit of a word from its isolated bit times the de Bruijn
// sequence 0x077CB531 (Leiserson, Prokop and Randall, 1998)
__constant__ unsigned char kLowBit[32] = {0, 1, 28, 2, 29, 14, 24, 3, 30, 22, 20, 15, 25, 17, 4, 8,
                                          31, 27, 13, 23, 21, 19, 16, 7, 26, 12, 18, 6, 11, 5, 10, 9};
using namespace dev;

// Bound of one wait for a chunk's bulk copy.  A copy of a chunk takes
// microseconds; a wait that runs out marks the tile stalled, counts it in
// g_waitStalls and ends the tile without output (ktmCheckDeviceWaits reports it).
constexpr unsigned long long kBulkWaitNs = 1000000000ull;
__device__ unsigned g_waitStalls;

// Per-CTA state of the chunk pipeline: one mbarrier per trace-row buffer.
struct ChunkSync {
    unsigned long long bar[2];
    int stalled;
};
static_assert(sizeof(ChunkSync) + sizeof(FastArgs) + sizeof(int) <= 1024,
              "static shared memory of the fast kernels within the 1 KB allowance");

struct ChunkSmem {
    // layout of one CTA's dynamic shared memory
    size_t rawBytes, crdOff, wtabOff, total;
};

// table: the kernel interpolates sqrt(j dt) from a per-CTA table (the table weight);
// the prefolded and sqrt.approx weights need none, and their chunks grow by its size
__host__ __device__ __forceinline__ ChunkSmem chunk_layout(int chunk, int pitch, int esize, int nt,
                                                           bool table)
{
    ChunkSmem L;
    L.rawBytes = (size_t)chunk * pitch * esize;              // one buffer
    L.crdOff = 2 * L.rawBytes;                               // [2][5][chunk] floats
    L.wtabOff = L.crdOff + ((2 * 5 * (size_t)chunk * 4 + 15) / 16) * 16;
    L.total = L.wtabOff + (table ? (size_t)(nt + 1) * sizeof(float2) : 0);   // [nt+1] weight table
    return L;
}

// Weight sqrt(t) of each pair (PRE):
//   kWtTable   sqrt(j dt) and its forward difference from a per-CTA table,
//              interpolated with the pair's own fraction f: relative error
//              about 1/(32 j^2), far below FP32 interpolation noise for j > 10;
//   kWtPrefold samples prefolded with sqrt(j dt) by ktmPrepareTraces: one
//              multiply less per pair, but the interpolation of the product
//              differs from the reference weight by f(1-f) dg dd (about 6e-4
//              relative L2 on shallow band-limited data), so it is opt-in;
//   kWtSqrt    a third sqrt.approx per pair on the special-function unit.
constexpr int kWtTable = 0, kWtPrefold = 1, kWtSqrt = 2;

// Output of a tile: the image (overwrite or accumulate), one trace slice's partial
// image, or atomic adds into the image (tiles of the batched launch).
enum { kOutImage = 0, kOutPartial = 1, kOutAtomic = 2 };

// One CTA-tile of the gather: image columns [colGroup*W, colGroup*W+W) x the tau
// run runIdx x traces [kb, ke), W = SH::kWarps.  Used by the grid launch (one tile
// per CTA) and by the persistent batched launch (a queue of tiles from many jobs).
template <class SH, int R, int PICK, int FMT, int PRE, int GRAD>
__device__ __forceinline__ bool fast_tile(const FastArgs& a, int chunk, int colGroup, int runIdx,
                                          int kb, int ke, float* __restrict__ partial, int outMode,
                                          unsigned char* smem_raw, ChunkSync& cs)
{
    static_assert(R % 2 == 0, "R pairs");
    using T = typename Elem<FMT>::T;
    const Geometry& g = a.g;
    const ChunkSmem L = chunk_layout(chunk, a.pitch, sizeof(T), a.g.nt, PRE == kWtTable);
    T* rawBase = reinterpret_cast<T*>(smem_raw);
    float* crdBase = reinterpret_cast<float*>(smem_raw + L.crdOff);
    float2* wtab = reinterpret_cast<float2*>(smem_raw + L.wtabOff);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncols = g.nx * g.ny;
    const int col = colGroup * SH::kWarps + warp;
    const bool colValid = col < ncols;
    const int ci = colValid ? col / g.ny : 0, cj = colValid ? col % g.ny : 0;
    const int run0 = runIdx * (32 * R);
    const float invdt = 1.0f / g.dt;

    // ---- per-thread tau tables, two tau samples per packed register pair ----
    f2 T2[R / 2], S2[R / 2], acc[R / 2];
    float t2min = 3.0e38f, smin = 3.0e38f;
    int nvalid = 0;
#pragma unroll
    for (int h = 0; h < R / 2; h++) {
        float tv[2], sv[2];
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int l = run0 + lane + 32 * (2 * h + e);
            const bool ok = l < g.nz;
            const int lc = ok ? l : g.nz - 1;
            const float tq = (g.z0 + (float)lc * g.dz) * invdt;
            const float v = a.velCube ? a.vel[(size_t)(colValid ? col : 0) * g.nz + lc] : a.vel[lc];
            const float vd = v * g.dt;
            tv[e] = tq * tq;
            sv[e] = 1.0f / (vd * vd);
            if (ok) { t2min = fminf(t2min, tv[e]); smin = fminf(smin, sv[e]); nvalid++; }
        }
        T2[h] = pk(tv[0], tv[1]);
        S2[h] = pk(sv[0], sv[1]);
        acc[h] = pk(0.0f, 0.0f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t2min = fminf(t2min, __shfl_xor_sync(0xffffffffu, t2min, o));
        smin = fminf(smin, __shfl_xor_sync(0xffffffffu, smin, o));
        nvalid += __shfl_xor_sync(0xffffffffu, nvalid, o);
    }
    const float colX = g.x0 + (float)ci * g.dx, colY = g.y0 + (float)cj * g.dy;
    if (PRE == kWtTable) {
        for (int j = threadIdx.x; j <= g.nt; j += SH::kThreads) {
            const float w0 = sqrtf((float)j * g.dt), w1 = sqrtf((float)(j + 1) * g.dt);
            wtab[j] = make_float2(w0, w1 - w0);
        }
    }

    const int nchunks = ke > kb ? (ke - kb + chunk - 1) / chunk : 0;
    const size_t rowBytes = (size_t)a.pitch * sizeof(T);

    auto issue = [&](int ch) {
        const int k0 = kb + ch * chunk, n = min(chunk, ke - k0);
        const int b = ch & 1;
        unsigned char* dst = reinterpret_cast<unsigned char*>(rawBase) + b * L.rawBytes;
        const unsigned char* src = static_cast<const unsigned char*>(a.traces) + (size_t)k0 * rowBytes;
        if (threadIdx.x == 0) bulk_g2s(dst, src, (unsigned)((size_t)n * rowBytes), &cs.bar[b]);
        float* crd = crdBase + b * 5 * chunk;
        for (int q = threadIdx.x; q < 5 * n; q += SH::kThreads) {
            const int arr = q / n, c = q % n;
            const float* srcArr = arr == 0 ? a.midX : arr == 1 ? a.midY : arr == 2 ? a.offX
                                : arr == 3 ? a.offY : a.scale;
            cp_async4(crd + arr * chunk + c, srcArr + k0 + c);
        }
        cp_async_commit();
    };

    const float umax = (float)g.nt;
    const float ap2 = a.aperture > 0.0f ? a.aperture * a.aperture : -1.0f;
    const f2 M2 = pk(kMagic, kMagic);
    unsigned keptTraces = 0;        // traces this warp evaluated (all lanes agree)

    // thread 0 owns both barriers: it arms them, waits on them and invalidates them
    if (threadIdx.x == 0) {
        mbar_init(&cs.bar[0], 1);
        mbar_init(&cs.bar[1], 1);
        cs.stalled = 0;
    }
    if (nchunks > 0) issue(0);
    for (int ch = 0; ch < nchunks; ch++) {
        const int b = ch & 1;
        const int k0 = kb + ch * chunk, n = min(chunk, ke - k0);
        cp_async_wait_all();
        // the ch/2-th use of buffer b completes phase ch/2 of its barrier
        if (threadIdx.x == 0 && !mbar_wait_bounded(&cs.bar[b], (ch >> 1) & 1, kBulkWaitNs)) {
            cs.stalled = 1;
            atomicAdd(&g_waitStalls, 1u);
            mbar_wait_bounded(&cs.bar[b], (ch >> 1) & 1, kBulkWaitNs);   // the copy in flight
        }
        __syncthreads();                       // chunk ch landed; chunk ch-1 fully consumed
        if (cs.stalled) return false;          // CTA-uniform: no output from this tile
        if (ch + 1 < nchunks) issue(ch + 1);
        if (colValid) {
            // ---- lane c: trace c's distances, scale and skip flag for this column ----
            // (chunk <= 32); the warp then walks the kept traces in increasing c,
            // taking their values by shuffle: no shared table, no second barrier
            const float* crd = crdBase + b * 5 * chunk;
            float lds_ = 0.0f, ldr_ = 0.0f, lsc = 0.0f;
            bool keep = false;
            if (lane < n) {
                const float mx = crd[lane], my = crd[chunk + lane], ox = crd[2 * chunk + lane],
                            oy = crd[3 * chunk + lane];
                lsc = crd[4 * chunk + lane];
                const float dmx = mx - colX, dmy = my - colY;
                const float sx = dmx - ox, sy = dmy - oy, rx = dmx + ox, ry = dmy + oy;
                lds_ = fmaf(sx, sx, sy * sy);           // explicit fusions: the same
                ldr_ = fmaf(rx, rx, ry * ry);           // values in every build
                keep = !(ap2 >= 0.0f && fmaf(dmx, dmx, dmy * dmy) > ap2);
                if (keep) {
                    // lower bound of u over the run: past the last sample -> no contribution
                    // approximate square roots: the margin below covers their error
                    const float ulb = sqrt_approx(fmaf(lds_, smin, t2min)) +
                                      sqrt_approx(fmaf(ldr_, smin, t2min));
                    keep = ulb < umax * 1.0001f + 1.0f;
                }
            }
            const unsigned rowsS = smem_u32(reinterpret_cast<const unsigned char*>(rawBase) + b * L.rawBytes);
            // bits(fl) = kMagicBits + i0: fold the magic offset into the bases (mod 2^32)
            const unsigned magicT = (unsigned)kMagicBits * (unsigned)sizeof(T);
            const unsigned wS = smem_u32(wtab) - (unsigned)kMagicBits * 8u;
            for (unsigned kept = __ballot_sync(0xffffffffu, keep); kept; kept &= kept - 1u) {
                // lowest kept trace: __ffs at 16 samples a lane, a de Bruijn lookup
                // (integer multiply, shift, constant table) for shorter runs; 8192 traces,
                // 512 / 384 / 256-sample runs: 201.3 / 211.5 / 221.3 ms with __ffs,
                // 202.1 / 202.6 / 218.5 with the lookup
                const int c = R == 16 ? __ffs(kept) - 1
                                      : (int)kLowBit[((kept & (0u - kept)) * 0x077CB531u) >> 27];
                const float ds = __shfl_sync(0xffffffffu, lds_, c);
                const float dr = __shfl_sync(0xffffffffu, ldr_, c);
                const float sc = __shfl_sync(0xffffffffu, lsc, c);
                keptTraces++;
                const unsigned rowS = rowsS + (unsigned)(c * a.pitch) * (unsigned)sizeof(T) - magicT;
                const f2 DS = pk(ds, ds), DR = pk(dr, dr), SC = pk(sc, sc);
#pragma unroll
                for (int h = 0; h < R / 2; h++) {
                    if (GRAD) {
                        // d/dS' of |tau| s_k W(u) V(u), u = sqrt(a_s) + sqrt(a_r):
                        // (dW/du V + W dV/du) du/dS', du/dS' = Ds/(2 sqrt a_s) + Dr/(2 sqrt a_r)
                        float as0, as1, ar0, ar1;
                        upk(fma2(DS, S2[h], T2[h]), as0, as1);
                        upk(fma2(DR, S2[h], T2[h]), ar0, ar1);
                        const f2 RS = pk(fminf(rsqrt_approx(as0), 3.0e38f), fminf(rsqrt_approx(as1), 3.0e38f));
                        const f2 RR = pk(fminf(rsqrt_approx(ar0), 3.0e38f), fminf(rsqrt_approx(ar1), 3.0e38f));
                        f2 U = fma2(pk(ar0, ar1), RR, mul2(pk(as0, as1), RS));
                        float u0, u1;
                        upk(U, u0, u1);
                        u0 = fminf(u0, umax);
                        u1 = fminf(u1, umax);
                        U = pk(u0, u1);
                        const f2 FL = add2_rm(U, M2);
                        float fl0, fl1;
                        upk(FL, fl0, fl1);
                        const unsigned q0 = __float_as_uint(fl0), q1 = __float_as_uint(fl1);
                        const f2 F = sub2(U, sub2(FL, M2));
                        const f2 DUDS = mul2(pk(0.5f, 0.5f), fma2(DS, RS, mul2(DR, RR)));
                        float a0, b0, a1, b1;
                        Lds<FMT>::pair(rowS + q0 * (unsigned)sizeof(T), a0, b0);
                        Lds<FMT>::pair(rowS + q1 * (unsigned)sizeof(T), a1, b1);
                        const f2 A = pk(a0, a1);
                        const f2 DV = sub2(pk(b0, b1), A);
                        f2 TERM;
                        if (PRE == kWtPrefold) {
                            TERM = DV;
                        } else {
                            const float2 w0 = lds_f2(wS + q0 * 8u), w1 = lds_f2(wS + q1 * 8u);
                            const f2 DW = pk(w0.y, w1.y);
                            const f2 W = fma2(F, DW, pk(w0.x, w1.x));
                            const f2 V = fma2(F, DV, A);
                            TERM = fma2(DW, V, mul2(W, DV));
                        }
                        acc[h] = fma2(mul2(SC, TERM), DUDS, acc[h]);
                        continue;
                    }
                    const PairKin kk = pair_kin(DS, DR, S2[h], T2[h], umax, M2);
                    const f2 F = kk.F;
                    const float u0 = kk.u0, u1 = kk.u1;
                    const unsigned q0 = kk.q0, q1 = kk.q1;
                    const unsigned ad0 = rowS + q0 * (unsigned)sizeof(T);
                    const unsigned ad1 = rowS + q1 * (unsigned)sizeof(T);
                    f2 V;
                    if (PICK == KTM_PICK_LINEAR) {
                        float a0, b0, a1, b1;
                        Lds<FMT>::pair(ad0, a0, b0);
                        Lds<FMT>::pair(ad1, a1, b1);
                        const f2 A = pk(a0, a1);
                        V = fma2(F, sub2(pk(b0, b1), A), A);
                    } else {
                        V = pk(Lds<FMT>::one(ad0), Lds<FMT>::one(ad1));
                    }
                    if (PRE == kWtPrefold) {
                        acc[h] = fma2(SC, V, acc[h]);
                    } else if (PRE == kWtTable) {
                        const float2 w0 = lds_f2(wS + q0 * 8u), w1 = lds_f2(wS + q1 * 8u);
                        const f2 W = fma2(F, pk(w0.y, w1.y), pk(w0.x, w1.x));
                        acc[h] = fma2(mul2(SC, W), V, acc[h]);
                    } else {
                        // u is in samples: sqrt(t) = sqrt(u) sqrt(dt), sqrt(dt) applied at the end
                        const f2 W = pk(sqrt_approx(u0), sqrt_approx(u1));
                        acc[h] = fma2(mul2(SC, W), V, acc[h]);
                    }
                }
            }
        }
    }

    if (threadIdx.x == 0) {
        mbar_inval(&cs.bar[0]);
        mbar_inval(&cs.bar[1]);
    }
    if (colValid) {
        float* out = (outMode == kOutPartial ? partial : a.image) + (size_t)col * g.nz;
#pragma unroll
        for (int h = 0; h < R / 2; h++) {
            float v2[2], s2[2];
            upk(acc[h], v2[0], v2[1]);
            upk(S2[h], s2[0], s2[1]);
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int l = run0 + lane + 32 * (2 * h + e);
                if (l < g.nz) {
                    const float tau = fabsf(g.z0 + (float)l * g.dz);
                    // GRAD: dI/dv = dI/dS' dS'/dv, S' = 1/(v dt)^2, dS'/dv = -2 dt S'^(3/2)
                    const float gfac = GRAD ? -2.0f * g.dt * s2[e] * sqrtf(s2[e]) : 1.0f;
                    const float v = v2[e] * gfac * (PRE == kWtSqrt ? tau * sqrtf(g.dt) : tau);
                    if (outMode == kOutAtomic) atomicAdd(out + l, v);
                    else out[l] = (outMode == kOutImage && a.accumulate) ? out[l] + v : v;
                }
            }
        }
    }
    if (a.pairsEvaluated && lane == 0 && keptTraces)
        atomicAdd(a.pairsEvaluated, (unsigned long long)keptTraces * (unsigned long long)nvalid);
    return true;
}

// ---------------------------------------------------------------------------
// Persistent batched launch: one CTA per SM slot pulls (job, column group, tau
// run, trace slice) tiles from a queue sorted longest first; each tile adds its
// result into its job's image with atomics (the images start at zero).  The
// job's arguments are copied into shared memory for the tile.
// ---------------------------------------------------------------------------
struct BatchTile {
    int job, cg, run, kb, ke, pad;
};

template <class SH, int R, int PICK, int FMT, int PRE>
__global__ void __launch_bounds__(SH::kThreads, SH::kMinBlocks)
batch_kernel(const FastArgs* __restrict__ jobs, const int* __restrict__ chunks,
             const BatchTile* __restrict__ tiles, int ntiles, unsigned* __restrict__ counter)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChunkSync cs;
    __shared__ FastArgs sa;
    __shared__ int st;
    static_assert(sizeof(FastArgs) % 4 == 0, "word copy");
    for (;;) {
        if (threadIdx.x == 0) st = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = st;
        if (t >= ntiles) break;                    // every thread read the same t
        const BatchTile tl = tiles[t];
        const int* src = reinterpret_cast<const int*>(jobs + tl.job);
        int* dst = reinterpret_cast<int*>(&sa);
        for (int i = threadIdx.x; i < (int)(sizeof(FastArgs) / 4); i += SH::kThreads) dst[i] = src[i];
        __syncthreads();
        const bool ok = fast_tile<SH, R, PICK, FMT, PRE, 0>(sa, chunks[tl.job], tl.cg, tl.run, tl.kb, tl.ke,
                                                        nullptr, kOutAtomic, smem_raw, cs);
        __syncthreads();                           // shared memory is reused by the next tile
        if (!ok) break;                            // CTA-uniform
    }
}

template <class SH, int R, int PICK, int FMT, int PRE, int GRAD>
__global__ void __launch_bounds__(SH::kThreads, SH::kMinBlocks)
fast_kernel(FastArgs a, int chunk, int perSlice, float* __restrict__ partial)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChunkSync cs;
    const int kb = blockIdx.z * perSlice;
    const int ke = min(a.g.ntr, kb + perSlice);
    const size_t nimg = (size_t)a.g.nx * a.g.ny * a.g.nz;
    fast_tile<SH, R, PICK, FMT, PRE, GRAD>(a, chunk, blockIdx.x, blockIdx.y, kb, ke,
                                       partial ? partial + blockIdx.z * nimg : nullptr,
                                       partial ? kOutPartial : kOutImage, smem_raw, cs);
}

// out[i] = (accumulate ? out[i] : 0) + sum_z partial[z][i], z in increasing order
__global__ void reduce_slices(float* __restrict__ out, const float* __restrict__ partial,
                              size_t nimg, int nslices, int accumulate)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nimg;
         i += (size_t)gridDim.x * blockDim.x) {
        float s = accumulate ? out[i] : 0.0f;
        for (int z = 0; z < nslices; z++) s += partial[(size_t)z * nimg + i];
        out[i] = s;
    }
}

// Traces per chunk: as many as the shape's shared-memory budget holds (at most
// kMaxChunk), or fewer when the caller caps them (chunkCap > 0).  0 when even one
// trace exceeds the largest allocation a CTA can have.
template <class SH>
int fast_chunk(const FastArgs& a, int esize, bool table)
{
    int chunk = kMaxChunk;
    if (a.chunkCap > 0) chunk = std::min(chunk, a.chunkCap);
    while (chunk > 1 && chunk_layout(chunk, a.pitch, esize, a.g.nt, table).total > SH::kBudget)
        chunk--;
    if (chunk_layout(chunk, a.pitch, esize, a.g.nt, table).total > (size_t)kMaxSmemBytes)
        return 0;
    return chunk;
}

// One grid launch over all of a's traces.
template <class SH, int R, int PICK, int FMT, int PRE, int GRAD>
int launch_block(const FastArgs& a, cudaStream_t stream, int smCount)
{
    const Geometry& g = a.g;
    const int esize = FMT == KTM_FMT_F32 ? 4 : 2;
    constexpr bool kTable = PRE == kWtTable;
    const int chunk = fast_chunk<SH>(a, esize, kTable);
    if (chunk == 0)
        return set_error(KTM_ERR_LIMIT, "fast kernel: packed pitch %d exceeds the shared-memory "
                                        "stage limit", a.pitch);
    const size_t smem = chunk_layout(chunk, a.pitch, esize, g.nt, kTable).total;
    auto kern = fast_kernel<SH, R, PICK, FMT, PRE, GRAD>;
    KTM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));

    const long long cols = (long long)g.nx * g.ny;
    const unsigned gx = (unsigned)((cols + SH::kWarps - 1) / SH::kWarps);
    const unsigned gy = (unsigned)((g.nz + 32 * R - 1) / (32 * R));
    if (gy > 65535) return set_error(KTM_ERR_LIMIT, "fast kernel: Nz too large");
    // trace slices: about eight CTAs per SM over the launch, each slice keeping at
    // least four chunks of traces
    const long long base = (long long)gx * gy;
    const long long want = 8LL * smCount;
    int slices = (int)((want + base - 1) / base);
    const int maxSlices = max(1, g.ntr / (4 * chunk));
    slices = max(1, min(slices, min(maxSlices, 64)));
    if (a.slices > 0) slices = min(a.slices, max(1, g.ntr));
    const int perSlice = (g.ntr + slices - 1) / slices;
    slices = (g.ntr + perSlice - 1) / perSlice;

    float* partial = nullptr;
    const size_t nimg = (size_t)cols * g.nz;
    if (slices > 1) {
        if (a.scratch && a.scratchBytes >= (size_t)slices * nimg * sizeof(float)) {
            partial = static_cast<float*>(a.scratch);
        } else {
            KTM_CUDA_TRY(pool_malloc(reinterpret_cast<void**>(&partial),
                                         (size_t)slices * nimg * sizeof(float), stream));
        }
    }
    dim3 grid(gx, gy, (unsigned)slices);
    kern<<<grid, SH::kThreads, smem, stream>>>(a, chunk, perSlice, partial);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && partial) {
        const int th = 256;
        const size_t want = (nimg + th - 1) / th, cap = (size_t)smCount * 8;
        const unsigned blocks = (unsigned)(want < cap ? want : cap);
        reduce_slices<<<blocks, th, 0, stream>>>(a.image, partial, nimg, slices, a.accumulate);
        e = cudaGetLastError();
    }
    if (partial && partial != a.scratch) cudaFreeAsync(partial, stream);
    if (e != cudaSuccess) return set_error(KTM_ERR_CUDA, "fast kernel launch: %s", cudaGetErrorString(e));
    return KTM_OK;
}

// Packed trace bytes per launch.  Every CTA streams all traces of its launch
// and CTAs start at different times, so the traces of one launch should stay
// resident in L2 (126 MB) while they are read: a trace set larger than this
// goes in blocks, one launch each, the later ones accumulating.
constexpr size_t kTraceBlockBytes = 40u << 20;

template <class SH, int R, int PICK, int FMT, int PRE, int GRAD>
int launch_t(const FastArgs& a, cudaStream_t stream, int smCount)
{
    const int esize = FMT == KTM_FMT_F32 ? 4 : 2;
    const size_t rowBytes = (size_t)a.pitch * esize;
    const int block = (int)std::max<size_t>(1024, kTraceBlockBytes / rowBytes);
    if (a.g.ntr <= block) return launch_block<SH, R, PICK, FMT, PRE, GRAD>(a, stream, smCount);
    // balanced blocks of at most `block` traces
    const int nblk = (a.g.ntr + block - 1) / block;
    const int per = (a.g.ntr + nblk - 1) / nblk;
    for (int kb = 0; kb < a.g.ntr; kb += per) {
        FastArgs b = a;
        b.g.ntr = std::min(per, a.g.ntr - kb);
        b.midX = a.midX + kb; b.midY = a.midY + kb; b.offX = a.offX + kb; b.offY = a.offY + kb;
        b.traces = static_cast<const unsigned char*>(a.traces) + (size_t)kb * rowBytes;
        b.scale = a.scale ? a.scale + kb : nullptr;
        b.accumulate = a.accumulate || kb > 0;
        const int rc = launch_block<SH, R, PICK, FMT, PRE, GRAD>(b, stream, smCount);
        if (rc) return rc;
    }
    return KTM_OK;
}

template <class SH, int R, int PICK, int PRE, int GRAD = 0>
int launch_fmt(const FastArgs& a, cudaStream_t s, int sm)
{
    switch (a.fmt) {
        case KTM_FMT_F32: return launch_t<SH, R, PICK, KTM_FMT_F32, PRE, GRAD>(a, s, sm);
        case KTM_FMT_F16: return launch_t<SH, R, PICK, KTM_FMT_F16, PRE, GRAD>(a, s, sm);
        default: return launch_t<SH, R, PICK, KTM_FMT_BF16, PRE, GRAD>(a, s, sm);
    }
}

// The paths a reduced shape is built for: linear pick, prefolded samples or the
// table weight, no gradient.
bool tunable_path(const FastArgs& a)
{
    return !a.grad && a.pick == KTM_PICK_LINEAR &&
           (a.weightMode == 2 || a.weightMethod == KTM_WEIGHT_TABLE);
}

template <class SH, int R>
int launch_pick(const FastArgs& a, cudaStream_t s, int sm)
{
    if constexpr (!SH::kFull) {
        if (!tunable_path(a))
            return set_error(KTM_ERR_ARG, "fast kernel: tileCols %d is built for the linear pick "
                                          "with the prefolded or table weight only (0 or 24 "
                                          "takes every path)", SH::kWarps);
        return a.weightMode == 2 ? launch_fmt<SH, R, KTM_PICK_LINEAR, kWtPrefold>(a, s, sm)
                                 : launch_fmt<SH, R, KTM_PICK_LINEAR, kWtTable>(a, s, sm);
    } else {
        if (a.grad) {
            // velocity gradient: linear pick; table weight or prefolded samples
            if (a.pick != KTM_PICK_LINEAR || (a.weightMode != 2 && a.weightMethod != KTM_WEIGHT_TABLE))
                return set_error(KTM_ERR_ARG, "ktmVrmsGradient takes the linear pick with the table "
                                              "weight or prefolded samples");
            return a.weightMode == 2 ? launch_fmt<SH, R, KTM_PICK_LINEAR, kWtPrefold, 1>(a, s, sm)
                                     : launch_fmt<SH, R, KTM_PICK_LINEAR, kWtTable, 1>(a, s, sm);
        }
        // a.weightMode: 2 samples prefolded; otherwise a.weightMethod picks table / sqrt
        if (a.weightMode == 2) {
            if (a.pick != KTM_PICK_LINEAR)
                return set_error(KTM_ERR_ARG, "truncating pick takes traces without the sqrt(t) fold");
            return launch_fmt<SH, R, KTM_PICK_LINEAR, kWtPrefold>(a, s, sm);
        }
        const bool sq = a.weightMethod == KTM_WEIGHT_SQRT;
        if (a.pick == KTM_PICK_LINEAR)
            return sq ? launch_fmt<SH, R, KTM_PICK_LINEAR, kWtSqrt>(a, s, sm)
                      : launch_fmt<SH, R, KTM_PICK_LINEAR, kWtTable>(a, s, sm);
        return sq ? launch_fmt<SH, R, KTM_PICK_TRUNCATE, kWtSqrt>(a, s, sm)
                  : launch_fmt<SH, R, KTM_PICK_TRUNCATE, kWtTable>(a, s, sm);
    }
}

template <class SH>
int launch_run(const FastArgs& a, int R, cudaStream_t s, int sm)
{
    switch (R) {
        case 8: return launch_pick<SH, 8>(a, s, sm);
        case 12: return launch_pick<SH, 12>(a, s, sm);
        case 16: return launch_pick<SH, 16>(a, s, sm);
        default: return set_error(KTM_ERR_ARG, "fast kernel: tileRun must be 256, 384 or 512");
    }
}

// tau samples per lane: from tileRun, or the run of 512 / 384 / 256 wasting the
// fewest samples at the end of Nz
int choose_run(int tileRun, int nz)
{
    if (tileRun > 0) return tileRun / 32;
    int best = 16, bestWaste = 1 << 30;
    for (int r : {16, 12, 8}) {
        const int run = 32 * r, waste = ((nz + run - 1) / run) * run - nz;
        if (waste < bestWaste) { bestWaste = waste; best = r; }
    }
    return best;
}

// ---------------------------------------------------------------------------
// FP64 device reference: one thread per image sample, traces straight from
// global memory.  Slow; used to measure the error of the fast path on
// configurations too large for the CPU oracle.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double load_any(const void* p, int fmt, size_t idx)
{
    if (fmt == KTM_FMT_F64) return static_cast<const double*>(p)[idx];
    if (fmt == KTM_FMT_F32) return (double)static_cast<const float*>(p)[idx];
    if (fmt == KTM_FMT_F16) return (double)__half2float(static_cast<const __half*>(p)[idx]);
    return (double)__bfloat162float(static_cast<const __nv_bfloat16*>(p)[idx]);
}

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
    const int stride = a.pitch;
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
        const size_t base = (size_t)k * stride;
        double val;
        if (a.pick == KTM_PICK_LINEAR) {
            const double fl = floor(u);
            const int i0 = (int)fl;
            const double f = u - fl;
            double d0 = (i0 > 0 && i0 < g.nt) ? load_any(a.traces, a.fmt, base + i0) : 0.0;
            double d1 = (i0 + 1 > 0 && i0 + 1 < g.nt) ? load_any(a.traces, a.fmt, base + i0 + 1) : 0.0;
            if (a.weightMode == 1) {
                d0 *= sqrt((double)i0 * dt);
                d1 *= sqrt((double)(i0 + 1) * dt);
            }
            val = (1.0 - f) * d0 + f * d1;
        } else {
            const int it = (int)u;
            val = (it > 0 && it < g.nt) ? load_any(a.traces, a.fmt, base + it) : 0.0;
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
    if (g.nt >= (1 << 22)) return set_error(KTM_ERR_LIMIT, "fast kernel: tracePts must be < 4194304");
    if (g.ntr == 0) {
        if (!a.accumulate)
            KTM_CUDA_TRY(cudaMemsetAsync(a.image, 0, sizeof(float) * (size_t)g.nx * g.ny * g.nz, stream));
        return KTM_OK;
    }
    const int esize = a.fmt == KTM_FMT_F32 ? 4 : 2;
    if (a.pitch < g.nt + 2 || ((size_t)a.pitch * esize) % 16 != 0 ||
        reinterpret_cast<uintptr_t>(a.traces) % 16 != 0)
        return set_error(KTM_ERR_ARG, "fast kernel: traces must be a packed set (pitch >= tracePts+2, "
                                      "16-byte rows, 16-byte aligned)");
    int dev = 0, sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    const int R = choose_run(a.tileRun, g.nz);
    switch (a.tileCols) {
        case 0:
        case 24: return launch_run<Shape24>(a, R, stream, sm);
        case 12: return launch_run<Shape12>(a, R, stream, sm);
        case 8: return launch_run<Shape8>(a, R, stream, sm);
        default: return set_error(KTM_ERR_ARG, "fast kernel: tileCols must be 0, 8, 12 or 24");
    }
}

int launch_f64_columns(const FastArgs& a, const int* cols, int ncols, double* out, cudaStream_t stream)
{
    const long long n = (long long)ncols * a.g.nz;
    if (n == 0) return KTM_OK;
    const int th = 128;
    f64_kernel<<<(unsigned)((n + th - 1) / th), th, 0, stream>>>(a, cols, ncols, out);
    KTM_CUDA_TRY(cudaGetLastError());
    return KTM_OK;
}

}  // namespace ktm

namespace ktm {
namespace {

template <class SH, int R, int PICK, int FMT, int PRE>
int launch_batch_t(const FastArgs* jobs, int njobs, cudaStream_t s)
{
    const int esize = FMT == KTM_FMT_F32 ? 4 : 2;
    int dev = 0, sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev);
    const int ctas = SH::kMinBlocks * sm;
    std::vector<int> chunks(njobs);
    size_t smem = 0;
    double totalPairs = 0.0;
    for (int j = 0; j < njobs; j++) {
        const Geometry& g = jobs[j].g;
        const int c = fast_chunk<SH>(jobs[j], esize, PRE == kWtTable);
        if (c == 0)
            return set_error(KTM_ERR_LIMIT, "batch: job %d packed pitch %d exceeds shared memory", j,
                             jobs[j].pitch);
        const size_t need = chunk_layout(c, jobs[j].pitch, esize, g.nt, PRE == kWtTable).total;
        chunks[j] = c;
        smem = std::max(smem, need);
        totalPairs += (double)g.nx * g.ny * g.nz * g.ntr;
    }
    // tiles: every job's column groups x tau runs, traces sliced so that no tile
    // exceeds ~1/16 of a CTA's share of the whole batch
    const double perTile = std::max(1.0, totalPairs / (ctas * 16.0));
    std::vector<BatchTile> tiles;
    std::vector<double> cost;
    for (int j = 0; j < njobs; j++) {
        const Geometry& g = jobs[j].g;
        const long long cols = (long long)g.nx * g.ny;
        if (cols * g.nz == 0 || g.ntr == 0) continue;
        const int cgs = (int)((cols + SH::kWarps - 1) / SH::kWarps);
        const int runs = (g.nz + 32 * R - 1) / (32 * R);
        const double tilePairsPerTrace = (double)SH::kWarps * 32 * R;
        int per = (int)std::min<double>(g.ntr, std::max<double>(4.0 * chunks[j], perTile / tilePairsPerTrace));
        per = std::max(per, 1);
        for (int cg = 0; cg < cgs; cg++)
            for (int r = 0; r < runs; r++)
                for (int kb = 0; kb < g.ntr; kb += per) {
                    const int ke = std::min(g.ntr, kb + per);
                    tiles.push_back(BatchTile{j, cg, r, kb, ke, 0});
                    cost.push_back(tilePairsPerTrace * (ke - kb));
                }
    }
    for (int j = 0; j < njobs; j++) {
        const Geometry& g = jobs[j].g;
        const size_t nimg = (size_t)g.nx * g.ny * g.nz;
        if (nimg) KTM_CUDA_TRY(cudaMemsetAsync(jobs[j].image, 0, nimg * sizeof(float), s));
    }
    if (tiles.empty()) return KTM_OK;
    // longest first, so that the queue's tail is made of short tiles
    std::vector<int> order(tiles.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    std::vector<BatchTile> sorted(tiles.size());
    for (size_t i = 0; i < order.size(); i++) sorted[i] = tiles[order[i]];

    const size_t bJobs = sizeof(FastArgs) * njobs, bChunks = sizeof(int) * njobs;
    const size_t bTiles = sizeof(BatchTile) * sorted.size();
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    unsigned char* buf = nullptr;
    KTM_CUDA_TRY(pool_malloc(reinterpret_cast<void**>(&buf), up(bJobs) + up(bChunks) + up(bTiles) + 256, s));
    FastArgs* dJobs = reinterpret_cast<FastArgs*>(buf);
    int* dChunks = reinterpret_cast<int*>(buf + up(bJobs));
    BatchTile* dTiles = reinterpret_cast<BatchTile*>(buf + up(bJobs) + up(bChunks));
    unsigned* dCounter = reinterpret_cast<unsigned*>(buf + up(bJobs) + up(bChunks) + up(bTiles));
    cudaError_t e = cudaMemcpyAsync(dJobs, jobs, bJobs, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dChunks, chunks.data(), bChunks, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dTiles, sorted.data(), bTiles, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dCounter, 0, sizeof(unsigned), s);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(batch_kernel<SH, R, PICK, FMT, PRE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
        const int grid = (int)std::min<size_t>((size_t)ctas, sorted.size());
        batch_kernel<SH, R, PICK, FMT, PRE><<<grid, SH::kThreads, smem, s>>>(dJobs, dChunks, dTiles,
                                                                      (int)sorted.size(), dCounter);
        e = cudaGetLastError();
    }
    // the host vectors above are pageable: these copies completed before returning
    cudaFreeAsync(buf, s);
    if (e != cudaSuccess) return set_error(KTM_ERR_CUDA, "batch launch: %s", cudaGetErrorString(e));
    return KTM_OK;
}

template <class SH, int R, int PICK, int PRE>
int launch_batch_fmt(const FastArgs* jobs, int n, cudaStream_t s)
{
    switch (jobs[0].fmt) {
        case KTM_FMT_F32: return launch_batch_t<SH, R, PICK, KTM_FMT_F32, PRE>(jobs, n, s);
        case KTM_FMT_F16: return launch_batch_t<SH, R, PICK, KTM_FMT_F16, PRE>(jobs, n, s);
        default: return launch_batch_t<SH, R, PICK, KTM_FMT_BF16, PRE>(jobs, n, s);
    }
}

template <class SH, int R>
int launch_batch_r(const FastArgs* jobs, int n, cudaStream_t s)
{
    const FastArgs& a = jobs[0];
    if constexpr (!SH::kFull) {
        if (!tunable_path(a))
            return set_error(KTM_ERR_ARG, "batch: tileCols %d is built for the linear pick with the "
                                          "prefolded or table weight only", SH::kWarps);
        return a.weightMode == 2 ? launch_batch_fmt<SH, R, KTM_PICK_LINEAR, kWtPrefold>(jobs, n, s)
                                 : launch_batch_fmt<SH, R, KTM_PICK_LINEAR, kWtTable>(jobs, n, s);
    } else {
        if (a.weightMode == 2) {
            if (a.pick != KTM_PICK_LINEAR)
                return set_error(KTM_ERR_ARG, "truncating pick takes traces without the sqrt(t) fold");
            return launch_batch_fmt<SH, R, KTM_PICK_LINEAR, kWtPrefold>(jobs, n, s);
        }
        const bool sq = a.weightMethod == KTM_WEIGHT_SQRT;
        if (a.pick == KTM_PICK_LINEAR)
            return sq ? launch_batch_fmt<SH, R, KTM_PICK_LINEAR, kWtSqrt>(jobs, n, s)
                      : launch_batch_fmt<SH, R, KTM_PICK_LINEAR, kWtTable>(jobs, n, s);
        return sq ? launch_batch_fmt<SH, R, KTM_PICK_TRUNCATE, kWtSqrt>(jobs, n, s)
                  : launch_batch_fmt<SH, R, KTM_PICK_TRUNCATE, kWtTable>(jobs, n, s);
    }
}

template <class SH>
int launch_batch_shape(const FastArgs* jobs, int n, int R, cudaStream_t s)
{
    switch (R) {
        case 8: return launch_batch_r<SH, 8>(jobs, n, s);
        case 12: return launch_batch_r<SH, 12>(jobs, n, s);
        case 16: return launch_batch_r<SH, 16>(jobs, n, s);
        default: return set_error(KTM_ERR_ARG, "batch: tileRun must be 256, 384 or 512");
    }
}

}  // namespace

int launch_batch(const FastArgs* jobs, int njobs, cudaStream_t s)
{
    if (njobs <= 0) return KTM_OK;
    const FastArgs& a = jobs[0];
    for (int j = 0; j < njobs; j++) {
        const FastArgs& b = jobs[j];
        if (b.fmt != a.fmt || b.pick != a.pick || b.weightMode != a.weightMode ||
            b.weightMethod != a.weightMethod)
            return set_error(KTM_ERR_ARG, "batch: every job needs the same trace format, pick and weight");
        const int esize = b.fmt == KTM_FMT_F32 ? 4 : 2;
        if (b.g.ntr > 0 && (b.pitch < b.g.nt + 2 || ((size_t)b.pitch * esize) % 16 != 0 ||
                            reinterpret_cast<uintptr_t>(b.traces) % 16 != 0))
            return set_error(KTM_ERR_ARG, "batch: job %d traces are not a packed set", j);
        if (b.g.nt >= (1 << 22)) return set_error(KTM_ERR_LIMIT, "batch: tracePts too large");
    }
    int R = a.tileRun > 0 ? a.tileRun / 32 : 0;
    if (R == 0) {
        int best = 16, bestWaste = 1 << 30;
        for (int r : {16, 12, 8}) {
            long long waste = 0;
            for (int j = 0; j < njobs; j++) {
                const int run = 32 * r, nz = jobs[j].g.nz;
                waste += (long long)(((nz + run - 1) / run) * run - nz) * jobs[j].g.nx * jobs[j].g.ny;
            }
            if (waste < bestWaste) { bestWaste = (int)std::min<long long>(waste, 1 << 30); best = r; }
        }
        R = best;
    }
    switch (a.tileCols) {
        case 0:
        case 24: return launch_batch_shape<Shape24>(jobs, njobs, R, s);
        case 12: return launch_batch_shape<Shape12>(jobs, njobs, R, s);
        case 8: return launch_batch_shape<Shape8>(jobs, njobs, R, s);
        default: return set_error(KTM_ERR_ARG, "batch: tileCols must be 0, 8, 12 or 24");
    }
}

namespace {

// One CTA bulk-copies `bytes` into shared memory and sums the landed words into
// out[0].  With stall = 1 thread 0 first waits on a second barrier that nothing
// arrives on: the wait runs out after limitNs and is counted in g_waitStalls,
// then the thread waits (bounded) for its own copy as a stalled tile does.
__global__ void wait_selftest_kernel(const unsigned* __restrict__ src, unsigned bytes, int stall,
                                     unsigned long long limitNs, unsigned* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char buf[];
    __shared__ unsigned long long bar[2];
    __shared__ int landed;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        bulk_g2s(buf, src, bytes, &bar[0]);
        if (stall && !mbar_wait_bounded(&bar[1], 0, limitNs)) atomicAdd(&g_waitStalls, 1u);
        landed = mbar_wait_bounded(&bar[0], 0, limitNs) ? 1 : 0;
        if (!landed) atomicAdd(&g_waitStalls, 1u);
        mbar_inval(&bar[0]);
        mbar_inval(&bar[1]);
    }
    __syncthreads();
    if (!landed) return;
    const unsigned* w = reinterpret_cast<const unsigned*>(buf);
    unsigned sum = 0;
    for (unsigned i = threadIdx.x; i < bytes / 4; i += blockDim.x) sum += w[i];
    atomicAdd(out, sum);
}

}  // namespace

int take_wait_stalls(cudaStream_t s, bool deviceSync, unsigned* n)
{
    unsigned v = 0;
    if (deviceSync) KTM_CUDA_TRY(cudaDeviceSynchronize());
    KTM_CUDA_TRY(cudaMemcpyFromSymbolAsync(&v, g_waitStalls, sizeof(v), 0, cudaMemcpyDeviceToHost, s));
    KTM_CUDA_TRY(cudaStreamSynchronize(s));
    if (v) {
        static const unsigned zero = 0;
        KTM_CUDA_TRY(cudaMemcpyToSymbolAsync(g_waitStalls, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s));
        KTM_CUDA_TRY(cudaStreamSynchronize(s));
    }
    *n = v;
    return KTM_OK;
}

int wait_selftest(int stall, unsigned long long limitNs, unsigned* checksum)
{
    constexpr unsigned kBytes = 64 * 1024, kWords = kBytes / 4;
    cudaStream_t s = 0;
    void* mem = nullptr;
    KTM_CUDA_TRY(pool_malloc(&mem, kBytes + 64, s));
    unsigned* src = static_cast<unsigned*>(mem);
    unsigned* out = src + kWords;
    int rc = KTM_OK;
    cudaError_t e = cudaMemsetAsync(src, 0x01, kBytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, 64, s);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(wait_selftest_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, kBytes);
    if (e == cudaSuccess) {
        wait_selftest_kernel<<<1, 256, kBytes, s>>>(src, kBytes, stall, limitNs, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(checksum, out, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = set_error(KTM_ERR_CUDA, "wait self-test: %s", cudaGetErrorString(e));
    cudaFreeAsync(mem, s);
    return rc;
}

}  // namespace ktm
