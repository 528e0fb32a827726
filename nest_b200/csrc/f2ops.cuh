// Packed FP32x2 arithmetic for sm_100 (FFMA2 / FADD2 / FMUL2 and the
// sub.f32x2 form): one instruction issue for a pair of FP32 values.  Used by
// the FP32 form's kernels, which are compiled with -use_fast_math (rcp2 and
// rsq2 are single MUFU operations per element).
#pragma once

#include <cuda_runtime.h>

namespace nestb {

using F2 = float2;

__device__ __forceinline__ F2 sp(float a) { return make_float2(a, a); }
__device__ __forceinline__ F2 add2(F2 a, F2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
    F2 o;
    asm("{\n\t.reg .b64 ta, tb, tr;\n\tmov.b64 ta, {%2, %3};\n\tmov.b64 tb, {%4, %5};\n\t"
        "sub.rn.f32x2 tr, ta, tb;\n\tmov.b64 {%0, %1}, tr;\n\t}"
        : "=f"(o.x), "=f"(o.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return o;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ F2 rcp2(F2 a) { return make_float2(__fdividef(1.f, a.x), __fdividef(1.f, a.y)); }
__device__ __forceinline__ F2 rsq2(F2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ F2 max2(F2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }
__device__ __forceinline__ F2 vmin2(F2 a, F2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ F2 vmax2(F2 a, F2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
// per-element select: c ? a : b
__device__ __forceinline__ F2 sel2(bool cx, bool cy, F2 a, F2 b) { return make_float2(cx ? a.x : b.x, cy ? a.y : b.y); }

}  // namespace nestb
