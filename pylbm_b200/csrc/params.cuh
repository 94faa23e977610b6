// Kernel-side view of an LbmDesc (validated on the host before any launch).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pylbm_b200.h"

namespace lbm {

struct StepParams {
    int n[3];      // nx, ny, nz (nz = 1 in 2D)
    int N;         // nodes
    int per[3];    // 1 if the axis is periodic (unused axes count as periodic)
    float ulid;    // lid speed (0 = no lid)
    float F[3];    // uniform force
    float r0, r1, r2, r3;
    const uint32_t* solid;  // optional 1-bit-per-node solid mask
    const float* field;     // optional per-node force (d, N)
    double* mx;             // optional momentum-exchange accumulator [d]
    const float* inlet;     // optional velocity inlet u_x(y) on the left wall (D2Q9)
    int outlet;             // 1: pressure outlet on the right boundary (D2Q9)
};

inline StepParams make_params(const LbmDesc& d) {
    StepParams p;
    p.n[0] = d.nx;
    p.n[1] = d.ny;
    p.n[2] = d.lattice == LBM_D2Q9 ? 1 : d.nz;
    p.N = p.n[0] * p.n[1] * p.n[2];
    const int dim = d.lattice == LBM_D2Q9 ? 2 : 3;
    for (int a = 0; a < 3; ++a) p.per[a] = (a >= dim) ? 1 : ((d.periodic_mask >> a) & 1);
    p.ulid = d.ulid;
    p.F[0] = d.fx;
    p.F[1] = d.fy;
    p.F[2] = dim == 3 ? d.fz : 0.0f;
    p.r0 = d.r0;
    p.r1 = d.r1;
    p.r2 = d.r2;
    p.r3 = d.r3;
    p.solid = d.solid_bits;
    p.field = d.force_field;
    p.mx = d.mx_force;
    p.inlet = d.inlet_u;
    p.outlet = d.outlet;
    return p;
}

__device__ __forceinline__ bool solid_at(const uint32_t* __restrict__ s, int n) {
    return (__ldg(s + (n >> 5)) >> (n & 31)) & 1u;
}

// Sum a double over the warp; lane 0 receives the total.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace lbm
