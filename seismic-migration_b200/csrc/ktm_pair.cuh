// ktm_pair.cuh -- device helpers shared by the gather kernels (migration,
// demigration, velocity gradient): packed f32x2 arithmetic, the special-function
// square root, shared-memory sample loads through 32-bit addresses, cp.async and
// bulk (TMA) copies with bounded mbarrier waits, and the per-pair kinematics, so
// that every operator evaluates the same traveltime, sample index, fraction and
// weight bit for bit.
#pragma once

#include "ktm_internal.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ktm {
namespace dev {

constexpr float kMagic = 12582912.0f;   // 1.5 * 2^23
constexpr int kMagicBits = 0x4B400000;

// ------------------------------------------------------------- f32x2 PTX ---
struct f2 {
    unsigned long long v;
};
__device__ __forceinline__ f2 pk(float a, float b)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void upk(f2 x, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(x.v));
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return r;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 add2_rm(f2 a, f2 b)
{
    f2 r;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
    return r;
}

__device__ __forceinline__ float rsqrt_approx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sqrt_approx(float x)
{
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// packed sample element -> float
template <int FMT> struct Elem;
template <> struct Elem<KTM_FMT_F32> {
    using T = float;
    static __device__ __forceinline__ float get(const T* p, int i) { return p[i]; }
};
template <> struct Elem<KTM_FMT_BF16> {
    using T = unsigned short;
    static __device__ __forceinline__ float get(const T* p, int i)
    {
        return __uint_as_float(static_cast<unsigned>(p[i]) << 16);
    }
};
template <> struct Elem<KTM_FMT_F16> {
    using T = __half;
    static __device__ __forceinline__ float get(const T* p, int i) { return __half2float(p[i]); }
};

// Shared-memory loads through 32-bit shared addresses.  The sample index comes
// out of the round-down magic add as bits(fl) = 0x4B400000 + i0, so the row
// base is pre-offset by -0x4B400000 * sizeof(T) (mod 2^32) and the address is
// one multiply-add of the float's bits.  Volatile: these loads must stay
// between the barriers that bracket each chunk.
template <int FMT> struct Lds;
template <> struct Lds<KTM_FMT_F32> {
    static __device__ __forceinline__ void pair(unsigned ad, float& a, float& b)
    {
        asm volatile("ld.shared.f32 %0, [%2];\n\tld.shared.f32 %1, [%2+4];" : "=f"(a), "=f"(b) : "r"(ad));
    }
    static __device__ __forceinline__ float one(unsigned ad)
    {
        float a;
        asm volatile("ld.shared.f32 %0, [%1];" : "=f"(a) : "r"(ad));
        return a;
    }
};
template <> struct Lds<KTM_FMT_BF16> {
    static __device__ __forceinline__ void pair(unsigned ad, float& a, float& b)
    {
        unsigned short x, y;
        asm volatile("ld.shared.u16 %0, [%2];\n\tld.shared.u16 %1, [%2+2];" : "=h"(x), "=h"(y) : "r"(ad));
        a = __uint_as_float(static_cast<unsigned>(x) << 16);
        b = __uint_as_float(static_cast<unsigned>(y) << 16);
    }
    static __device__ __forceinline__ float one(unsigned ad)
    {
        unsigned short x;
        asm volatile("ld.shared.u16 %0, [%1];" : "=h"(x) : "r"(ad));
        return __uint_as_float(static_cast<unsigned>(x) << 16);
    }
};
template <> struct Lds<KTM_FMT_F16> {
    static __device__ __forceinline__ void pair(unsigned ad, float& a, float& b)
    {
        unsigned short x, y;
        asm volatile("ld.shared.b16 %0, [%2];\n\tld.shared.b16 %1, [%2+2];" : "=h"(x), "=h"(y) : "r"(ad));
        a = __half2float(__ushort_as_half(x));
        b = __half2float(__ushort_as_half(y));
    }
    static __device__ __forceinline__ float one(unsigned ad)
    {
        unsigned short x;
        asm volatile("ld.shared.b16 %0, [%1];" : "=h"(x) : "r"(ad));
        return __half2float(__ushort_as_half(x));
    }
};
__device__ __forceinline__ float2 lds_f2(unsigned ad)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(ad));
    return v;
}
__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem)
{
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n"); }

// ---- bulk (TMA) copies global -> shared, completed on an mbarrier ----------
// One thread initialises, arms and waits on the barrier; a __syncthreads after
// its wait publishes the landed bytes to the rest of the CTA.
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned arrivals)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long* bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
// Arms the barrier for `bytes` and starts the copy.  dst, src and bytes are
// multiples of 16.  The proxy fence orders the CTA's earlier reads of dst
// (generic proxy) before the copy's writes (async proxy).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar)
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n"
                 " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase of the given parity to complete; false when limitNs of
// wall time passed first.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity,
                                                  unsigned long long limitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limitNs) return false;
    }
}


// Kinematics of two pairs (tau samples r and r+1 of one lane) with one trace:
//   a_s = T2' + Ds S', a_r = T2' + Dr S'   (sample units)
//   u   = min(sqrt(a_s) + sqrt(a_r), nt)   (NaN -> nt: a zero guard)
//   fl  = u + 1.5*2^23 rounded down: bits(fl) = 0x4B400000 + floor(u)
//   f   = u - floor(u)
struct PairKin {
    f2 U, F;
    float u0, u1;
    unsigned q0, q1;      // bits(fl): 0x4B400000 + floor(u)
};
__device__ __forceinline__ PairKin pair_kin(f2 DS, f2 DR, f2 S2, f2 T2, float umax, f2 M2)
{
    PairKin k;
    float as0, as1, ar0, ar1;
    upk(fma2(DS, S2, T2), as0, as1);
    upk(fma2(DR, S2, T2), ar0, ar1);
    f2 U = add2(pk(sqrt_approx(as0), sqrt_approx(as1)), pk(sqrt_approx(ar0), sqrt_approx(ar1)));
    upk(U, k.u0, k.u1);
    k.u0 = fminf(k.u0, umax);
    k.u1 = fminf(k.u1, umax);
    k.U = pk(k.u0, k.u1);
    const f2 FL = add2_rm(k.U, M2);
    float fl0, fl1;
    upk(FL, fl0, fl1);
    k.q0 = __float_as_uint(fl0);
    k.q1 = __float_as_uint(fl1);
    k.F = sub2(k.U, sub2(FL, M2));
    return k;
}

}  // namespace dev
}  // namespace ktm
