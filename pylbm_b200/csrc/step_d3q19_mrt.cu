// D3Q19 MRT (d'Humieres et al. 2002 basis) on the register row kernels: the AB pull and
// AA-odd row kernels of step_rows3d.cuh and the AA-even vector kernel, each colliding its
// lane's nodes in a rolled loop with one copy of the pair-folded moment transform
// (collide.cuh). A translation unit of its own so that it compiles beside step_d3q19.cu.
#include "dispatch.cuh"
#include "staged_launch.cuh"
#include "step_rows3d.cuh"

namespace lbm {
namespace {

using L = D3Q19;

template <int STORE, bool FORCE>
int go_mrt(const StepParams& P, const void* src, void* dst, int pattern, cudaStream_t s) {
    if (pattern == LBM_PATTERN_AA_EVEN) return go_aa_even<L, STORE, LBM_MRT, FORCE>(P, dst, s);
    if (pattern == LBM_PATTERN_AB) return rows3d::go_ab<STORE, LBM_MRT, FORCE>(P, src, dst, s);
    return rows3d::go_aa_odd<STORE, LBM_MRT, FORCE>(P, dst, s);
}

template <int STORE>
int go_mrt_f(const LbmDesc& d, const void* src, void* dst, int pattern, cudaStream_t s) {
    const StepParams P = make_params(d);
    return needs_force(d) ? go_mrt<STORE, true>(P, src, dst, pattern, s)
                          : go_mrt<STORE, false>(P, src, dst, pattern, s);
}

}  // namespace

int launch_mrt_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern,
                     cudaStream_t s) {
    switch (d.storage) {
        case LBM_STORE_F32: return go_mrt_f<LBM_STORE_F32>(d, src, dst, pattern, s);
        case LBM_STORE_F32_SHIFTED: return go_mrt_f<LBM_STORE_F32_SHIFTED>(d, src, dst, pattern, s);
        case LBM_STORE_F16: return go_mrt_f<LBM_STORE_F16>(d, src, dst, pattern, s);
        case LBM_STORE_BF16: return go_mrt_f<LBM_STORE_BF16>(d, src, dst, pattern, s);
    }
    return LBM_E_STORAGE;
}

}  // namespace lbm
