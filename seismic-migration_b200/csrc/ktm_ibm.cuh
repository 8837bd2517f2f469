// ktm_ibm.cuh -- IBM System/360 single precision to IEEE float on the device,
// the arithmetic of ktmIBM32toIEEE (ioFunctions.c:18-38) operation for
// operation, so that the result is bit-identical to the reference built for
// x86-64 (SSE, no contraction):
//
//   out = (sign * (fraction / 0xFFFFFF)) * 16^(exponent - 64)
//
// sign = -1 or 1 from bit 31, exponent = bits 30..24, fraction = bits 23..0.
// The fraction converts exactly (24 bits), the quotient is one correctly
// rounded division (FRACTION_MASK, not 2^24: a bias of 2^-24 the reference
// carries), and 16^e = 2^(4e) is built from its bits: a normal, a subnormal
// (4e in [-149, -127]), zero below, infinity above 127 -- the values powf
// returns for these exact powers.  The two products round to nearest even
// with subnormals kept (the library is built without flush-to-zero).
#pragma once

#include <cstdint>

namespace ktm {
namespace dev {

__device__ __forceinline__ float pow2_exact(int e)
{
    if (e > 127) return __int_as_float(0x7f800000);
    if (e >= -126) return __int_as_float((e + 127) << 23);
    if (e >= -149) return __int_as_float(1 << (e + 149));
    return 0.0f;
}

__device__ __forceinline__ float ibm32_to_f32(uint32_t w)
{
    const float sign = (w & 0x80000000u) ? -1.0f : 1.0f;
    const float q = __fdiv_rn(__uint2float_rn(w & 0x00ffffffu), 16777215.0f);
    const int e = (int)((w >> 24) & 127u) - 64;
    const float p = pow2_exact(4 * e);
    // 0 * inf: x86 SSE returns its default NaN (sign set, quiet bit set), which
    // is what the reference writes; the device's canonical NaN differs in bits.
    if (q == 0.0f && e * 4 > 127) return __int_as_float(0xffc00000);
    return __fmul_rn(__fmul_rn(sign, q), p);
}

}  // namespace dev
}  // namespace ktm
