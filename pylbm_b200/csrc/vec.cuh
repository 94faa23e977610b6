// 16-byte vectors of stored populations: 4 fp32 or 8 fp16 / bf16 elements per uint4.
//
// Elements are handled as raw bit patterns (uint32 holding 32 or 16 bits) so that the x-shift
// of a row segment is a register permutation plus one warp shuffle, independent of the type;
// conversion to fp32 happens once per node, right before the collision.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <cstring>

#include "../../include/pylbm_b200.h"

namespace lbm {

template <int STORE>
struct VT;

template <>
struct VT<LBM_STORE_F32> {
    using E = uint32_t;
    static constexpr int V = 4;
    __device__ __forceinline__ static float f(uint32_t b) { return __uint_as_float(b); }
    __device__ __forceinline__ static uint32_t b(float v) { return __float_as_uint(v); }
};
template <>
struct VT<LBM_STORE_F32_SHIFTED> : VT<LBM_STORE_F32> {};

template <>
struct VT<LBM_STORE_F16> {
    using E = uint16_t;
    static constexpr int V = 8;
    __device__ __forceinline__ static float f(uint32_t b) {
        return __half2float(__ushort_as_half(static_cast<unsigned short>(b)));
    }
    __device__ __forceinline__ static uint32_t b(float v) {
        return __half_as_ushort(__float2half_rn(v));
    }
};

template <>
struct VT<LBM_STORE_BF16> {
    using E = uint16_t;
    static constexpr int V = 8;
    __device__ __forceinline__ static float f(uint32_t b) { return __uint_as_float(b << 16); }
    __device__ __forceinline__ static uint32_t b(float v) {
        return __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
};

__device__ __forceinline__ uint32_t word(const uint4& v, int j) {
    return j == 0 ? v.x : (j == 1 ? v.y : (j == 2 ? v.z : v.w));
}
__device__ __forceinline__ void set_word(uint4& v, int j, uint32_t w) {
    if (j == 0) v.x = w;
    else if (j == 1) v.y = w;
    else if (j == 2) v.z = w;
    else v.w = w;
}

// element k (compile-time after unrolling) of a vector of V elements
template <int V>
__device__ __forceinline__ uint32_t elem(const uint4& v, int k) {
    if constexpr (V == 4) return word(v, k);
    else return (word(v, k >> 1) >> ((k & 1) * 16)) & 0xffffu;
}
template <int V>
__device__ __forceinline__ void put(uint4& v, int k, uint32_t e) {
    if constexpr (V == 4) {
        set_word(v, k, e);
    } else {
        const uint32_t w = word(v, k >> 1);
        set_word(v, k >> 1, (k & 1) ? ((w & 0x0000ffffu) | (e << 16)) : ((w & 0xffff0000u) | e));
    }
}

// Shift a vector by one element along x: shift_up gives element k = v[k - 1] and element 0 =
// `up`; shift_down gives element k = v[k + 1] and element V - 1 = `dn` (the new elements sit
// in the low bits of up / dn). For 16-bit elements each output word is one byte permutation
// of two input words.
template <int V>
__device__ __forceinline__ uint4 shift_up(const uint4& v, uint32_t up) {
    if constexpr (V == 4) {
        return make_uint4(up, v.x, v.y, v.z);
    } else {
        return make_uint4(__byte_perm(up, v.x, 0x5410), __byte_perm(v.x, v.y, 0x5432),
                          __byte_perm(v.y, v.z, 0x5432), __byte_perm(v.z, v.w, 0x5432));
    }
}
template <int V>
__device__ __forceinline__ uint4 shift_down(const uint4& v, uint32_t dn) {
    if constexpr (V == 4) {
        return make_uint4(v.y, v.z, v.w, dn);
    } else {
        return make_uint4(__byte_perm(v.x, v.y, 0x5432), __byte_perm(v.y, v.z, 0x5432),
                          __byte_perm(v.z, v.w, 0x5432), __byte_perm(v.w, dn, 0x5432));
    }
}

// Two 16-bit elements of one word <-> two floats (packed conversions).
template <int STORE>
__device__ __forceinline__ float2 unpack2(uint32_t w) {
    if constexpr (STORE == LBM_STORE_F16) {
        __half2 h;
        memcpy(&h, &w, 4);
        return __half22float2(h);
    } else {
        return make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u));
    }
}
template <int STORE>
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    uint32_t w;
    if constexpr (STORE == LBM_STORE_F16) {
        const __half2 h = __floats2half2_rn(lo, hi);
        memcpy(&w, &h, 4);
    } else {
        const __nv_bfloat162 b = __floats2bfloat162_rn(lo, hi);
        memcpy(&w, &b, 4);
    }
    return w;
}

// Whole-vector moves.
__device__ __forceinline__ uint4 ld_nc(const void* p) {
    return __ldg(reinterpret_cast<const uint4*>(p));
}
__device__ __forceinline__ uint4 ld_plain(const void* p) {
    return *reinterpret_cast<const uint4*>(p);
}
__device__ __forceinline__ void st_cs(void* p, const uint4& v) {
    __stcs(reinterpret_cast<uint4*>(p), v);
}
__device__ __forceinline__ void st_plain(void* p, const uint4& v) {
    *reinterpret_cast<uint4*>(p) = v;
}

// The elements 1..V-1 of vector u into p[1..V-1] (st_tail), or the elements 0..V-2 of d into
// p[0..V-2] (st_head), p 16-byte aligned: the other slot belongs to a node of another warp.
// Three aligned stores (16-bit: 2 + 4 + 8 bytes; fp32: 4 + 8) instead of V - 1 single ones.
template <int V, class E>
__device__ __forceinline__ void st_tail(E* p, const uint4& u) {
    if constexpr (V == 8) {
        *reinterpret_cast<uint16_t*>(p + 1) = static_cast<uint16_t>(u.x >> 16);
        *reinterpret_cast<uint32_t*>(p + 2) = u.y;
        *reinterpret_cast<uint2*>(p + 4) = make_uint2(u.z, u.w);
    } else {
        *reinterpret_cast<uint32_t*>(p + 1) = u.y;
        *reinterpret_cast<uint2*>(p + 2) = make_uint2(u.z, u.w);
    }
}
template <int V, class E>
__device__ __forceinline__ void st_head(E* p, const uint4& d) {
    if constexpr (V == 8) {
        *reinterpret_cast<uint2*>(p) = make_uint2(d.x, d.y);
        *reinterpret_cast<uint32_t*>(p + 4) = d.z;
        *reinterpret_cast<uint16_t*>(p + 6) = static_cast<uint16_t>(d.w & 0xffffu);
    } else {
        *reinterpret_cast<uint2*>(p) = make_uint2(d.x, d.y);
        *reinterpret_cast<uint32_t*>(p + 2) = d.z;
    }
}

// Single elements.
template <class E>
__device__ __forceinline__ uint32_t ld1_nc(const E* p) {
    return uint32_t(__ldg(p));
}
template <class E>
__device__ __forceinline__ uint32_t ld1(const E* p) {
    return uint32_t(*p);
}
template <class E>
__device__ __forceinline__ void st1(E* p, uint32_t e) {
    *p = static_cast<E>(e);
}

}  // namespace lbm
