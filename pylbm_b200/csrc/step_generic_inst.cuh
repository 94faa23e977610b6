// Template dispatch of the generic kernel for one lattice (included once per lattice).
#pragma once

#include "dispatch.cuh"
#include "step_generic.cuh"

namespace lbm {

template <class L, int COLL, int STORE, int PATTERN, bool FORCE>
static int go_generic(const StepParams& P, const void* src, void* dst, cudaStream_t s) {
    using T = typename Codec<STORE>::T;
    const int bx = block_x_for(P.n[0]);
    const dim3 grid((P.n[0] + bx - 1) / bx, P.n[1], P.n[2]);
    k_step_generic<L, COLL, STORE, PATTERN, FORCE>
        <<<grid, bx, 0, s>>>(P, static_cast<const T*>(src), static_cast<T*>(dst));
    return int(cudaGetLastError());
}

template <class L, int COLL, int STORE, int PATTERN>
static int go_force(const LbmDesc& d, const StepParams& P, const void* src, void* dst,
                    cudaStream_t s) {
    if (needs_force(d)) return go_generic<L, COLL, STORE, PATTERN, true>(P, src, dst, s);
    return go_generic<L, COLL, STORE, PATTERN, false>(P, src, dst, s);
}

template <class L, int COLL, int STORE>
static int go_pattern(const LbmDesc& d, const StepParams& P, const void* src, void* dst,
                      int pattern, cudaStream_t s) {
    switch (pattern) {
        case LBM_PATTERN_AB: return go_force<L, COLL, STORE, LBM_PATTERN_AB>(d, P, src, dst, s);
        case LBM_PATTERN_AA_ODD:
            return go_force<L, COLL, STORE, LBM_PATTERN_AA_ODD>(d, P, src, dst, s);
        case LBM_PATTERN_AA_EVEN:
            return go_force<L, COLL, STORE, LBM_PATTERN_AA_EVEN>(d, P, src, dst, s);
    }
    return LBM_E_PATTERN;
}

template <class L, int COLL>
static int go_storage(const LbmDesc& d, const StepParams& P, const void* src, void* dst,
                      int pattern, cudaStream_t s) {
    switch (d.storage) {
        case LBM_STORE_F32: return go_pattern<L, COLL, LBM_STORE_F32>(d, P, src, dst, pattern, s);
        case LBM_STORE_F16: return go_pattern<L, COLL, LBM_STORE_F16>(d, P, src, dst, pattern, s);
        case LBM_STORE_BF16:
            return go_pattern<L, COLL, LBM_STORE_BF16>(d, P, src, dst, pattern, s);
        case LBM_STORE_F32_SHIFTED:
            return go_pattern<L, COLL, LBM_STORE_F32_SHIFTED>(d, P, src, dst, pattern, s);
    }
    return LBM_E_STORAGE;
}

}  // namespace lbm
