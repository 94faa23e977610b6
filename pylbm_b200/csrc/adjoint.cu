// Adjoint of the D2Q9 BGK fused step with Guo forcing, walls, periodic axes and solids, for
// gradients of a momentum-exchange objective with respect to a per-node force field.
//
// Forward step (pull): f_{t+1}(x) = C_x(g(x); F(x)), g = P f_t, P = streaming with half-way
// bounce-back (walls, solids), C = BGK with Guo forcing:
//   rho = sum g, u = (sum c g + F/2) / rho,
//   p_i = g_i + w (feq_i - g_i) + (1 - w/2) S_i.
// Reverse step t (lambda_{t+1} = dJ/df_{t+1} known): mu_t = (dC/dg)^T lambda_{t+1} per node,
// dJ/dF(x) += (dC/dF)^T lambda_{t+1}, lambda_t = dPhi_t/df_t + P^T mu_t. With
//   L0 = sum_i lambda_i w_i, L1 = sum_i lambda_i w_i c_i, L2 = sum_i lambda_i w_i c_i c_i^T,
//   K  = 3 L1 + 9 L2 u - 3 L0 u,   T = (1 - w/2) (9 L2 F - 3 L0 F) / (2 rho),
//   A  = L0 (1 - 1.5 u.u) + 3 L1.u + 4.5 u^T L2 u,
// (from du/dg_j = (c_j - u) / rho, du/dF = I / (2 rho), dfeq_i/drho|_u = feq_i / rho) one gets
//   (dC/dF)^T lambda = K + T,
//   mu_j = (1 - w) lambda_j + w A + (w K + 2 T) . (c_j - u).
// So the reverse kernel needs only rho and u of the forward step, which the recomputation
// pass records (lbm_forward_record), not the populations. P^T (the transposed pull) reads
// mu at x + c_j when node x + c_j pulls direction j from x (link open, x fluid), or the node's
// own mu_opp(j) when that pull bounces back (x + c_j behind a wall or solid). The objective's
// derivative is added where the window weight is non-zero: dPhi/df_i(x) = 2 c_ix on fluid
// nodes whose neighbour x + c_i is solid (karman.py:45-53,88-96, np.roll wrap).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/pylbm_b200.h"
#include "codec.cuh"
#include "collide.cuh"
#include "dispatch.cuh"
#include "step_generic.cuh"

namespace lbm {
namespace {

using L = D2Q9;

// Forward BGK step that also writes the rho and u the collision used: ru = (rho, ux, uy)
// planes of N floats. Same pull and arithmetic as the generic kernel (shifted storages).
template <int STORE, bool FORCE>
__global__ void __launch_bounds__(128)
k_forward_record(const StepParams P, const typename Codec<STORE>::T* __restrict__ A,
                 typename Codec<STORE>::T* __restrict__ B, float* __restrict__ ru) {
    using C = Codec<STORE>;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= P.n[0]) return;
    const int y = blockIdx.y;
    const int crd[3] = {x, y, 0};
    const int n = x + P.n[0] * y;
    const int N = P.N;
    float h[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        int idx = i * N + n;
        bool top = false;
        if (i != 0) {
            bool wall;
            const int off = link<L>(P, crd, i, -1, wall, top);
            const bool blocked = wall || (P.solid != nullptr && solid_at(P.solid, n + off));
            idx = blocked ? L::opp(i) * N + n : i * N + n + off;
        }
        h[i] = C::ld(A[idx]);
        if (top && L::cx(i) != 0) h[i] = add_lid(h[i], lid_term<L>(i, P.ulid));
    }
    float F[3] = {P.F[0], P.F[1], 0.0f};
    if (FORCE && P.field != nullptr) {
        F[0] += __ldg(P.field + n);
        F[1] += __ldg(P.field + N + n);
    }
    float rho, u[3];
    collide<L, LBM_BGK, true, FORCE, C::compact, true>(h, F, P.r0, 0.0f, 0.0f, 0.0f, &rho, u);
    ru[n] = rho;
    ru[N + n] = u[0];
    ru[2 * N + n] = u[1];
#pragma unroll
    for (int i = 0; i < 9; ++i) B[i * N + n] = C::st(h[i]);
}

// One reverse step. mu_in = mu_{t+1} (NULL: zero, the last step), mu_out = mu_t,
// grad (2 N doubles) += (dC/dF)^T lambda_{t+1}; objw = weight of Phi_{t+1} in J (0 outside
// the averaging window).
__global__ void __launch_bounds__(128)
k_adjoint_bgk(const StepParams P, const float* __restrict__ ru, const float* __restrict__ mu_in,
              float* __restrict__ mu_out, double* __restrict__ grad, float objw) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= P.n[0]) return;
    const int y = blockIdx.y;
    const int crd[3] = {x, y, 0};
    const int n = x + P.n[0] * y;
    const int N = P.N;
    const bool fluid = P.solid == nullptr || !solid_at(P.solid, n);
    // ---------------------------------------------------------------- lambda_{t+1}
    float lam[9];
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        float v = 0.0f;
        if (mu_in != nullptr) {
            if (j == 0) {
                v = mu_in[n];  // the rest population never streams
            } else {
                bool wall, top;
                const int off = link<L>(P, crd, j, +1, wall, top);
                const bool blocked = wall || (P.solid != nullptr && solid_at(P.solid, n + off));
                if (blocked) v = mu_in[L::opp(j) * N + n];
                else if (fluid) v = mu_in[j * N + n + off];
            }
        }
        if (objw != 0.0f && j != 0 && L::cx(j) != 0 && fluid &&
            solid_at(P.solid, wrapped<L>(P, crd, j)))
            v += 2.0f * objw * float(L::cx(j));
        lam[j] = v;
    }
    // ---------------------------------------------------------------- transposed collision
    const float rho = ru[n], ux = ru[N + n], uy = ru[2 * N + n];
    float Fx = P.F[0], Fy = P.F[1];
    if (P.field != nullptr) {
        Fx += __ldg(P.field + n);
        Fy += __ldg(P.field + N + n);
    }
    float L0 = 0.0f, L1x = 0.0f, L1y = 0.0f, Lxx = 0.0f, Lxy = 0.0f, Lyy = 0.0f;
#pragma unroll
    for (int j = 0; j < 9; ++j) {
        const float lw = L::w(j) * lam[j];
        const float cx = float(L::cx(j)), cy = float(L::cy(j));
        L0 += lw;
        L1x += cx * lw;
        L1y += cy * lw;
        Lxx += cx * cx * lw;
        Lxy += cx * cy * lw;
        Lyy += cy * cy * lw;
    }
    const float om = P.r0;
    const float L2ux = Lxx * ux + Lxy * uy, L2uy = Lxy * ux + Lyy * uy;
    const float Kx = 3.0f * L1x + 9.0f * L2ux - 3.0f * L0 * ux;
    const float Ky = 3.0f * L1y + 9.0f * L2uy - 3.0f * L0 * uy;
    const float tf = (1.0f - 0.5f * om) / (2.0f * rho);
    const float Tx = tf * (9.0f * (Lxx * Fx + Lxy * Fy) - 3.0f * L0 * Fx);
    const float Ty = tf * (9.0f * (Lxy * Fx + Lyy * Fy) - 3.0f * L0 * Fy);
    const float usq = ux * ux + uy * uy;
    const float Av = L0 * (1.0f - 1.5f * usq) + 3.0f * (L1x * ux + L1y * uy) +
                     4.5f * (ux * L2ux + uy * L2uy);
    const float Bx = om * Kx + 2.0f * Tx, By = om * Ky + 2.0f * Ty;
    const float base = om * Av - (Bx * ux + By * uy);
#pragma unroll
    for (int j = 0; j < 9; ++j)
        mu_out[j * N + n] = (1.0f - om) * lam[j] + base + Bx * float(L::cx(j)) +
                            By * float(L::cy(j));
    grad[n] += double(Kx + Tx);
    grad[N + n] += double(Ky + Ty);
}

int check_adjoint_desc(const LbmDesc* d) {
    const int rc = lbm_validate(d);
    if (rc) return rc;
    if (d->lattice != LBM_D2Q9) return LBM_E_LATTICE;
    if (d->collision != LBM_BGK) return LBM_E_COLLISION;
    if (d->storage != LBM_STORE_F32_SHIFTED && d->storage != LBM_STORE_F16 &&
        d->storage != LBM_STORE_BF16)
        return LBM_E_STORAGE;
    return LBM_OK;
}

dim3 grid_of(const StepParams& P) { return dim3((P.n[0] + 127) / 128, P.n[1]); }

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" {

int lbm_forward_record(const LbmDesc* d, const void* src, void* dst, float* rho_u,
                       uint64_t stream) {
    int rc = check_adjoint_desc(d);
    if (rc) return rc;
    if (!src || !dst || !rho_u) return LBM_E_NULL;
    if (src == dst) return LBM_E_ALIAS;
    const StepParams P = make_params(*d);
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const bool force = needs_force(*d);
    switch (d->storage) {
        case LBM_STORE_F32_SHIFTED:
            if (force)
                k_forward_record<LBM_STORE_F32_SHIFTED, true><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const float*>(src), static_cast<float*>(dst), rho_u);
            else
                k_forward_record<LBM_STORE_F32_SHIFTED, false><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const float*>(src), static_cast<float*>(dst), rho_u);
            break;
        case LBM_STORE_F16:
            if (force)
                k_forward_record<LBM_STORE_F16, true><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const __half*>(src), static_cast<__half*>(dst), rho_u);
            else
                k_forward_record<LBM_STORE_F16, false><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const __half*>(src), static_cast<__half*>(dst), rho_u);
            break;
        default:
            if (force)
                k_forward_record<LBM_STORE_BF16, true><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const __nv_bfloat16*>(src), static_cast<__nv_bfloat16*>(dst),
                    rho_u);
            else
                k_forward_record<LBM_STORE_BF16, false><<<grid_of(P), 128, 0, s>>>(
                    P, static_cast<const __nv_bfloat16*>(src), static_cast<__nv_bfloat16*>(dst),
                    rho_u);
    }
    return int(cudaGetLastError());
}

int lbm_adjoint_step(const LbmDesc* d, const float* rho_u, const float* mu_in, float* mu_out,
                     double* grad, double objw, uint64_t stream) {
    int rc = check_adjoint_desc(d);
    if (rc) return rc;
    if (!rho_u || !mu_out || !grad) return LBM_E_NULL;
    if (mu_in == mu_out) return LBM_E_ALIAS;
    if (!std::isfinite(objw)) return LBM_E_ARG;
    if (objw != 0.0 && d->solid_bits == nullptr) return LBM_E_ARG;
    const StepParams P = make_params(*d);
    k_adjoint_bgk<<<grid_of(P), 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        P, rho_u, mu_in, mu_out, grad, float(objw));
    return int(cudaGetLastError());
}

}  // extern "C"
