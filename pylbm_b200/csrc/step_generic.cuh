// Generic fused stream-collide kernel: one lattice node per thread, every feature.
//
// This is the kernel for any shape and option set the specialised kernels do not cover
// (x extents that are not a multiple of the vector width, solids, per-node forces, the
// momentum-exchange reduction). It follows pylbm's pattern semantics (codegen.py:10-16):
//   ab      : read f[i, x - c_i] (bounce-back: f[opp(i), x]), collide, write g[i, x]
//   aa-odd  : read A[opp(i), x - c_i] (bounce-back: A[i, x]), collide,
//             write A[i, x + c_i] (bounce-back: A[opp(i), x] minus the lid term)
//   aa-even : read A[i, x], collide, write A[opp(i), x]
// Boundary precedence is core.py:88-127: a link that leaves the box through a wall bounces
// back from the node itself and, if it leaves through the top wall of the last axis, gains
// Ladd's moving-wall term +6 w_i c_ix U (pull) / -6 w_i c_ix U (AA push). Otherwise the
// source is wrapped on periodic axes, and a solid source node bounces back without a lid
// term (core.py:101-105).
#pragma once

#include "codec.cuh"
#include "collide.cuh"
#include "lattice.cuh"
#include "params.cuh"

namespace lbm {

// Resolve the node reached from crd along sign * c_i. Returns the flat offset to add to n
// and sets wall (the link crosses a non-periodic boundary) and top (it crosses the top wall
// of the last axis, where the lid sits).
template <class L>
__device__ __forceinline__ int link(const StepParams& P, const int (&crd)[3], int i, int sign,
                                    bool& wall, bool& top) {
    wall = false;
    top = false;
    int off = 0;
    int stride = 1;
#pragma unroll
    for (int a = 0; a < L::D; ++a) {
        const int c = sign * cc<L>(i, a);
        if (c != 0) {
            int s = crd[a] + c;
            if (s < 0 || s >= P.n[a]) {
                if (P.per[a]) {
                    s += (s < 0) ? P.n[a] : -P.n[a];
                } else {
                    wall = true;
                    if (a == L::D - 1 && s >= P.n[a]) top = true;
                }
            }
            off += (s - crd[a]) * stride;
        }
        stride *= P.n[a];
    }
    return off;
}

// Flat index of crd + c_i wrapped on EVERY axis (np.roll semantics), used for the solid
// lookups of the momentum-exchange masks (karman.py:45-53).
template <class L>
__device__ __forceinline__ int wrapped(const StepParams& P, const int (&crd)[3], int i) {
    int idx = 0;
    int stride = 1;
#pragma unroll
    for (int a = 0; a < L::D; ++a) {
        int s = crd[a] + cc<L>(i, a);
        s += (s < 0) ? P.n[a] : ((s >= P.n[a]) ? -P.n[a] : 0);
        idx += s * stride;
        stride *= P.n[a];
    }
    return idx;
}

// Velocity inlet on the left wall (core.py:67-78,116-117): a pull of direction i (c_ix = +1)
// at x = 0 bounces back with Ladd's term for the wall speed u_in(y), 6 w_i c_ix u_in(y),
// unless the source also lies behind a y wall, whose rule comes later in pylbm's axis loop
// and wins at the corners.
template <class L>
__device__ __forceinline__ void apply_inlet(const StepParams& P, int y, float (&f)[L::Q]) {
    const float uin = __ldg(P.inlet + y);
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
        if (L::cx(i) != 1) continue;
        const int ys = y - L::cy(i);
        if (!P.per[1] && (ys < 0 || ys >= P.n[1])) continue;
        f[i] = add_lid(f[i], __fmul_rn(6.0f * L::w(i) * float(L::cx(i)), uin));
    }
}

// Pressure outlet on the right boundary (core.py:130-148), applied after every other rule:
// the pulls with c_ix = -1 at x = nx - 1 take the equilibrium at rho = 1 and the velocity of
// the neighbouring column x = nx - 2 of the stored (pre-streaming) state, in pylbm's order of
// operations; shifted storages hold that equilibrium minus w_i.
template <class L, class C>
__device__ __forceinline__ void apply_outlet(const StepParams& P,
                                             const typename C::T* __restrict__ A, int n,
                                             float (&f)[L::Q]) {
    static_assert(L::Q == 9, "the outlet is defined for D2Q9");
    float col[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) col[i] = C::ld(A[i * P.N + n - 1]);
    float rho = col[0];
#pragma unroll
    for (int i = 1; i < 9; ++i) rho = rho + col[i];
    if (C::shifted) rho = 1.0f + rho;
    const float ux = (col[1] - col[3] + col[5] - col[6] - col[7] + col[8]) / rho;
    const float uy = (col[2] - col[4] + col[5] + col[6] - col[7] - col[8]) / rho;
    const float usq = ux * ux + uy * uy;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        if (L::cx(i) != -1) continue;
        const float cu = float(L::cx(i)) * ux + float(L::cy(i)) * uy;
        const float dev = 3.0f * cu + 4.5f * cu * cu - 1.5f * usq;
        f[i] = C::shifted ? L::w(i) * dev : L::w(i) * (1.0f + dev);
    }
}

template <class L, int COLL, int STORE, int PATTERN, bool FORCE>
__global__ void __launch_bounds__(128)
k_step_generic(const StepParams P, const typename Codec<STORE>::T* A,
               typename Codec<STORE>::T* B) {
    using C = Codec<STORE>;
    constexpr int Q = L::Q;
    constexpr bool SHIFT = C::shifted;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    const bool active = x < P.n[0];
    const int crd[3] = {active ? x : 0, y, z};
    const int n = crd[0] + P.n[0] * (y + P.n[1] * z);
    const int N = P.N;
    const bool has_solid = P.solid != nullptr;

    float f[Q];
    if (active) {
        // ------------------------------------------------------------ stream (pull)
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            int idx;
            bool top = false;
            if (PATTERN == LBM_PATTERN_AA_EVEN || i == 0) {
                idx = (PATTERN == LBM_PATTERN_AA_ODD ? L::opp(i) : i) * N + n;
            } else {
                bool wall;
                const int off = link<L>(P, crd, i, -1, wall, top);
                const bool blocked = wall || (has_solid && solid_at(P.solid, n + off));
                if (PATTERN == LBM_PATTERN_AB)
                    idx = blocked ? L::opp(i) * N + n : i * N + n + off;
                else
                    idx = blocked ? i * N + n : L::opp(i) * N + n + off;
            }
            f[i] = C::ld(A[idx]);
            if (top && L::cx(i) != 0) f[i] = add_lid(f[i], lid_term<L>(i, P.ulid));
        }
        if constexpr (L::D == 2 && PATTERN == LBM_PATTERN_AB) {  // open boundaries
            if (P.inlet != nullptr && x == 0) apply_inlet<L>(P, y, f);
            if (P.outlet && x == P.n[0] - 1) apply_outlet<L, C>(P, A, n, f);
        }
        // ------------------------------------------------------------ collide
        float F[3] = {P.F[0], P.F[1], P.F[2]};
        if (FORCE && P.field != nullptr) {
#pragma unroll
            for (int a = 0; a < L::D; ++a) F[a] += __ldg(P.field + a * N + n);
        }
        collide<L, COLL, SHIFT, FORCE, C::compact>(f, F, P.r0, P.r1, P.r2, P.r3);
    }

    // ---------------------------------------------------------------- momentum exchange
    if (PATTERN == LBM_PATTERN_AB && P.mx != nullptr) {
        double acc[3] = {0.0, 0.0, 0.0};
        if (active && !solid_at(P.solid, n)) {
#pragma unroll
            for (int i = 1; i < Q; ++i) {
                if (solid_at(P.solid, wrapped<L>(P, crd, i))) {
                    const double v = double(f[i]) + (SHIFT ? L::wd(i) : 0.0);
#pragma unroll
                    for (int a = 0; a < L::D; ++a) acc[a] += double(cc<L>(i, a)) * v;
                }
            }
        }
        const bool any = __any_sync(0xffffffffu, acc[0] != 0.0 || acc[1] != 0.0 || acc[2] != 0.0);
        if (any) {
#pragma unroll
            for (int a = 0; a < L::D; ++a) {
                const double s = warp_sum(acc[a]);
                if ((threadIdx.x & 31) == 0) atomicAdd(P.mx + a, 2.0 * s);
            }
        }
    }
    if (!active) return;

    // ---------------------------------------------------------------- write
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        if (PATTERN == LBM_PATTERN_AB) {
            B[i * N + n] = C::st(f[i]);
        } else if (PATTERN == LBM_PATTERN_AA_EVEN) {
            B[L::opp(i) * N + n] = C::st(f[i]);
        } else {
            if (i == 0) {
                B[n] = C::st(f[0]);
                continue;
            }
            bool wall, top;
            const int off = link<L>(P, crd, i, +1, wall, top);
            if (wall) {
                float v = f[i];
                if (top && L::cx(i) != 0) v = sub_lid(v, lid_term<L>(i, P.ulid));
                B[L::opp(i) * N + n] = C::st(v);
            } else {
                B[i * N + n + off] = C::st(f[i]);
            }
        }
    }
}

}  // namespace lbm
