// Generic kernel instantiations for D3Q19 (BGK, TRT, MRT).
#include "step_generic_inst.cuh"

namespace lbm {

int launch_generic_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern,
                         cudaStream_t s) {
    const StepParams P = make_params(d);
    switch (d.collision) {
        case LBM_BGK: return go_storage<D3Q19, LBM_BGK>(d, P, src, dst, pattern, s);
        case LBM_TRT: return go_storage<D3Q19, LBM_TRT>(d, P, src, dst, pattern, s);
        case LBM_MRT: return go_storage<D3Q19, LBM_MRT>(d, P, src, dst, pattern, s);
        case LBM_STREAM_ONLY:
            return go_storage<D3Q19, LBM_STREAM_ONLY>(d, P, src, dst, pattern, s);
    }
    return LBM_E_COLLISION;
}

}  // namespace lbm
