// Packed FP32 pairs (sm_100a `.f32x2` arithmetic).
//
// One instruction applies the same IEEE round-to-nearest operation to two
// independent floats held in a 64-bit register pair, so a pair of pixels
// that blend the same splat costs one issue slot per operation instead of
// two.  Each lane's result is bit-identical to the scalar `__fadd_rn` /
// `__fmul_rn` / `__fmaf_rn` of the same operands (no flush to zero: the
// `.ftz` modifier is not used).
#pragma once

#include <cstdint>

namespace gs {

using f2 = unsigned long long;  // {lo, hi} = {lane 0, lane 1}

__device__ __forceinline__ f2 f2_pack(const float lo, const float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 f2_dup(const float x) { return f2_pack(x, x); }
__device__ __forceinline__ void f2_unpack(const f2 v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 f2_add(const f2 a, const f2 b)
{
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_sub(const f2 a, const f2 b)
{
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 f2_mul(const f2 a, const f2 b)
{
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
// a * b + c with one rounding, per lane
__device__ __forceinline__ f2 f2_fma(const f2 a, const f2 b, const f2 c)
{
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

}  // namespace gs
