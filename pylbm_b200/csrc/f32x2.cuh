// Value types for the shifted collisions of the 16-bit storages.
//
// F2 holds the same quantity of two nodes (the two halves of one 32-bit storage word) and
// computes with sm_100's packed fp32 instructions (add / sub / mul / fma .rn.f32x2): one
// instruction for both nodes, each half rounded exactly as the scalar fp32 operation. The
// 16-bit kernels need twice the node rate of fp32 for the same bytes and are bound by
// instruction issue, so this halves their collision cost.
//
// F1 is one node with the same explicitly rounded operations (never contracted into fma,
// never reassociated), so a kernel that collides one node per thread (the generic, staged
// and adjoint-recording kernels, and the D3Q19 register kernels) produces bit-for-bit what
// the packed kernels produce.
//
// Plain float keeps the compiler's freedom (contraction) for the fp32 storages.
#pragma once

#include <cuda_runtime.h>

namespace lbm {

struct F1 {
    float v;
};
struct F2 {
    float2 v;
};

template <class S>
__device__ __forceinline__ S sc(float c);
template <>
__device__ __forceinline__ float sc<float>(float c) { return c; }
template <>
__device__ __forceinline__ F1 sc<F1>(float c) { return {c}; }
template <>
__device__ __forceinline__ F2 sc<F2>(float c) { return {make_float2(c, c)}; }

// ---------------------------------------------------------------------------- F1
__device__ __forceinline__ F1 operator+(F1 a, F1 b) { return {__fadd_rn(a.v, b.v)}; }
__device__ __forceinline__ F1 operator-(F1 a, F1 b) { return {__fsub_rn(a.v, b.v)}; }
__device__ __forceinline__ F1 operator*(F1 a, F1 b) { return {__fmul_rn(a.v, b.v)}; }
__device__ __forceinline__ F1 fma_(F1 a, F1 b, F1 c) { return {__fmaf_rn(a.v, b.v, c.v)}; }
// 1 / a for a near 1 (the density): the hardware approximation refined by one Newton-Raphson
// step, r' = r + r (1 - a r), three instructions without the slow-path branch of an IEEE
// reciprocal (the two agree to about an ulp; operands are never zero, infinite or subnormal)
__device__ __forceinline__ float rcp_nr(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    const float e = __fmaf_rn(-a, r, 1.0f);
    return __fmaf_rn(r, e, r);
}
__device__ __forceinline__ F1 rcp_(F1 a) { return {rcp_nr(a.v)}; }

// ---------------------------------------------------------------------------- F2
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 fma_(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {  // no intrinsic: sub.rn.f32x2
    unsigned long long ra, rb, rd;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.v.x), "f"(a.v.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.v.x), "f"(b.v.y));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    F2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.v.x), "=f"(d.v.y) : "l"(rd));
    return d;
}
__device__ __forceinline__ F2 rcp_(F2 a) {
    return {make_float2(rcp_nr(a.v.x), rcp_nr(a.v.y))};
}

// ---------------------------------------------------------------------------- float
__device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float rcp_(float a) { return __frcp_rn(a); }

// 1 + x and -x, per node with scalar instructions (an immediate operand instead of a
// broadcast constant pair); rounded alike (or exact) for all three types.
__device__ __forceinline__ float one_plus(float x) { return 1.0f + x; }
__device__ __forceinline__ F1 one_plus(F1 x) { return {__fadd_rn(1.0f, x.v)}; }
__device__ __forceinline__ F2 one_plus(F2 x) {
    return {make_float2(__fadd_rn(1.0f, x.v.x), __fadd_rn(1.0f, x.v.y))};
}
__device__ __forceinline__ float neg_(float x) { return -x; }
__device__ __forceinline__ F1 neg_(F1 x) { return {-x.v}; }
__device__ __forceinline__ F2 neg_(F2 x) { return {make_float2(-x.v.x, -x.v.y)}; }

// The scalar value of a one-node type (for the optional rho / u outputs).
__device__ __forceinline__ float scalar_of(float a) { return a; }
__device__ __forceinline__ float scalar_of(F1 a) { return a.v; }

}  // namespace lbm
