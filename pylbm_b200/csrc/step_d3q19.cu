// D3Q19 specialised kernels: register row kernels for the AB pull and the AA-odd step (the
// default), the TMA-staged kernel for both with LBM_FLAG_STAGED, vector AA-even.
#include "codec.cuh"
#include "collide.cuh"
#include "dispatch.cuh"
#include "staged_launch.cuh"
#include "step_rows3d.cuh"
#include "step_staged_rows.cuh"

namespace lbm {
namespace {

using L = D3Q19;

template <int STORE, int COLL, bool FORCE>
int go(const StepParams& P, const void* src, void* dst, int pattern, cudaStream_t s,
       bool staged) {
    if (pattern == LBM_PATTERN_AA_EVEN) return go_aa_even<L, STORE, COLL, FORCE>(P, dst, s);
    if (pattern == LBM_PATTERN_AB) {
        if constexpr (STORE == LBM_STORE_F16 || STORE == LBM_STORE_BF16) {
            if (staged) {  // whole periodic rows: the row-staged kernel; else the segment one
                const int rc = go_staged_rows16<STORE, COLL, FORCE>(P, src, dst, s);
                if (rc != 1) return rc;
            }
        }
        if (staged) return go_staged<L, STORE, COLL, FORCE, LBM_PATTERN_AB>(P, src, dst, s);
        return rows3d::go_ab<STORE, COLL, FORCE>(P, src, dst, s);
    }
    if (staged) return go_staged<L, STORE, COLL, FORCE, LBM_PATTERN_AA_ODD>(P, dst, dst, s);
    return rows3d::go_aa_odd<STORE, COLL, FORCE>(P, dst, s);
}

template <int STORE, int COLL>
int go_f(const LbmDesc& d, const StepParams& P, const void* src, void* dst, int pattern,
         cudaStream_t s) {
    const bool staged = (d.flags & LBM_FLAG_STAGED) != 0;
    return needs_force(d) ? go<STORE, COLL, true>(P, src, dst, pattern, s, staged)
                          : go<STORE, COLL, false>(P, src, dst, pattern, s, staged);
}

template <int STORE>
int go_c(const LbmDesc& d, const StepParams& P, const void* src, void* dst, int pattern,
         cudaStream_t s) {
    switch (d.collision) {
        case LBM_BGK: return go_f<STORE, LBM_BGK>(d, P, src, dst, pattern, s);
        case LBM_TRT: return go_f<STORE, LBM_TRT>(d, P, src, dst, pattern, s);
        // MRT: the register row kernels with a rolled node loop, in a translation unit of
        // their own (step_d3q19_mrt.cu); no TMA-staged form
        case LBM_MRT: return launch_mrt_d3q19(d, src, dst, pattern, s);
        case LBM_STREAM_ONLY:
            return go<STORE, LBM_STREAM_ONLY, false>(P, src, dst, pattern, s,
                                                     (d.flags & LBM_FLAG_STAGED) != 0);
    }
    return LBM_E_COLLISION;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

int launch_staged_timeout_probe(const LbmDesc& d, void* buf, unsigned long long timeout_ns,
                                cudaStream_t s) {
    const StepParams P = make_params(d);
    return go_staged<L, LBM_STORE_F32_SHIFTED, LBM_BGK, false, LBM_PATTERN_AB>(
        P, buf, buf, s, /*no_issue=*/1, timeout_ns);
}

int launch_fast_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern,
                      cudaStream_t s) {
    if (d.solid_bits || d.force_field || d.mx_force || d.inlet_u || d.outlet) return 1;
    const int V = (d.storage == LBM_STORE_F16 || d.storage == LBM_STORE_BF16) ? 8 : 4;
    if (d.nx % V != 0) return 1;
    if (!aligned16(src) || !aligned16(dst)) return 1;
    const StepParams P = make_params(d);
    switch (d.storage) {
        case LBM_STORE_F32: return go_c<LBM_STORE_F32>(d, P, src, dst, pattern, s);
        case LBM_STORE_F32_SHIFTED: return go_c<LBM_STORE_F32_SHIFTED>(d, P, src, dst, pattern, s);
        case LBM_STORE_F16: return go_c<LBM_STORE_F16>(d, P, src, dst, pattern, s);
        case LBM_STORE_BF16: return go_c<LBM_STORE_BF16>(d, P, src, dst, pattern, s);
    }
    return LBM_E_STORAGE;
}

}  // namespace lbm
