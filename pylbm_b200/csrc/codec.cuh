// Storage codec: how a population is held in HBM and turned into fp32 for the arithmetic.
//
// pylbm's fused kernels hold either f in fp32 or the shifted value f - w_i in fp16 / bf16
// (lbm.cu:16-42, _fused.py:83-90). This library adds fp32 holding f - w_i. In every shifted
// storage the collision also computes on h = f - w_i (see collide.cuh), so the value read is
// used as is and the weight is never added back in fp32.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "../../include/pylbm_b200.h"

namespace lbm {

template <int STORE>
struct Codec;

template <>
struct Codec<LBM_STORE_F32> {
    using T = float;
    static constexpr bool shifted = false;
    static constexpr bool compact = false;  // 16-bit storage
    __device__ __forceinline__ static float ld(T v) { return v; }
    __device__ __forceinline__ static T st(float v) { return v; }
};

template <>
struct Codec<LBM_STORE_F32_SHIFTED> {
    using T = float;
    static constexpr bool shifted = true;
    static constexpr bool compact = false;
    __device__ __forceinline__ static float ld(T v) { return v; }
    __device__ __forceinline__ static T st(float v) { return v; }
};

template <>
struct Codec<LBM_STORE_F16> {
    using T = __half;
    static constexpr bool shifted = true;
    static constexpr bool compact = true;
    __device__ __forceinline__ static float ld(T v) { return __half2float(v); }
    __device__ __forceinline__ static T st(float v) { return __float2half_rn(v); }
};

template <>
struct Codec<LBM_STORE_BF16> {
    using T = __nv_bfloat16;
    static constexpr bool shifted = true;
    static constexpr bool compact = true;
    __device__ __forceinline__ static float ld(T v) { return __bfloat162float(v); }
    __device__ __forceinline__ static T st(float v) { return __float2bfloat16_rn(v); }
};

}  // namespace lbm
