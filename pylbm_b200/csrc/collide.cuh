// Node-local collision: moments, equilibrium, Guo source, BGK / TRT / MRT relaxation.
//
// The formulas are pylbm's (core.py:151-247, lbm.cu:100-163):
//   rho = sum f,  u = (sum c f + F/2) / rho                              (Guo half force)
//   feq_i = w_i rho (1 - 1.5 u.u + c_i.u (3 + 4.5 c_i.u))
//   S_i = w_i [3 (c_i.F - u.F) + 9 (c_i.u)(c_i.F)]
//   BGK: p_i = f_i + r0 (feq_i - f_i) + (1 - r0/2) S_i
//   TRT: symmetric / antisymmetric parts relaxed with r0 = s+ and r1 = s-, forcing split
//        the same way
//   MRT (D2Q9): dm_k = (-s_k [M (f - feq)]_k + (1 - s_k/2) [M S]_k) / |M_k|^2,
//               p = f + M^T dm, rates (0, r1, r2, 0, r3, 0, r3, r0, r0)
//
// Two arithmetic forms share this code:
//  * plain (SHIFT = false): the operands are f, evaluated in the order of lbm.cu so that the
//    fp32 result tracks pylbm's own CUDA C kernel;
//  * shifted (SHIFT = true): the operands are h = f - w_i. With drho = sum h, rho = 1 + drho,
//    sum w_i c_i = 0 and sum w_i = 1, every quantity above is rewritten without the O(w_i)
//    constant: heq_i = w_i (drho + rho (c_i.u (3 + 4.5 c_i.u) - 1.5 u.u)), and
//    f - feq = h - heq, so p - w = h + r0 (heq - h) + ... . fp32 rounding then acts on the
//    O(|h|) deviations only, which is what keeps 1000 fp32 steps within 1e-6 of float64.
#pragma once

#include "lattice.cuh"

namespace lbm {

// In: f[] pre-collision (h if SHIFT), F = total force at the node (zeros when unforced).
// Out: f[] post-collision (h* if SHIFT).
template <class L, int COLL, bool SHIFT, bool FORCE>
__device__ __forceinline__ void collide(float (&f)[L::Q], const float (&F)[3], float r0,
                                        float r1, float r2, float r3) {
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    if constexpr (COLL == LBM_STREAM_ONLY) return;  // debug mode: streaming only
    // ---------------------------------------------------------------- moments
    float rho_s = 0.0f;  // rho (plain) or drho (shifted)
#pragma unroll
    for (int i = 0; i < Q; ++i) rho_s += f[i];
    float j[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int a = 0; a < D; ++a) {
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const int c = cc<L>(i, a);
            if (c == 1) j[a] += f[i];
            if (c == -1) j[a] -= f[i];
        }
    }
    const float rho = SHIFT ? 1.0f + rho_s : rho_s;
    const float inv_rho = 1.0f / rho;
    float u[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int a = 0; a < D; ++a) u[a] = (FORCE ? j[a] + 0.5f * F[a] : j[a]) * inv_rho;
    float usq = u[0] * u[0];
#pragma unroll
    for (int a = 1; a < D; ++a) usq += u[a] * u[a];
    float uf = 0.0f;
    if (FORCE) {
        uf = u[0] * F[0];
#pragma unroll
        for (int a = 1; a < D; ++a) uf += u[a] * F[a];
    }

    // ---------------------------------------------------------------- equilibrium, source
    float feq[Q];
    float S[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        float cu = 0.0f, cf = 0.0f;
#pragma unroll
        for (int a = 0; a < D; ++a) {
            const int c = cc<L>(i, a);
            if (c == 1) { cu += u[a]; cf += F[a]; }
            if (c == -1) { cu -= u[a]; cf -= F[a]; }
        }
        const float wi = L::w(i);
        if (SHIFT) {
            feq[i] = wi * (rho_s + rho * (cu * (3.0f + 4.5f * cu) - 1.5f * usq));
        } else {
            feq[i] = wi * rho * (1.0f - 1.5f * usq + cu * (3.0f + 4.5f * cu));
        }
        S[i] = FORCE ? wi * (3.0f * (cf - uf) + 9.0f * cu * cf) : 0.0f;
    }

    // ---------------------------------------------------------------- relax
    if (COLL == LBM_BGK) {
        const float g = 1.0f - 0.5f * r0;
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            float p = f[i] + r0 * (feq[i] - f[i]);
            if (FORCE) p += g * S[i];
            f[i] = p;
        }
    } else if (COLL == LBM_TRT) {
        const float gp = 1.0f - 0.5f * r0;
        const float gm = 1.0f - 0.5f * r1;
        {
            float p = f[0] - r0 * (f[0] - feq[0]);
            if (FORCE) p += gp * S[0];
            f[0] = p;
        }
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            const int o = L::opp(i);
            if (o < i) continue;  // each opposite pair once
            const float np_ = 0.5f * (f[i] + f[o]) - 0.5f * (feq[i] + feq[o]);
            const float nm_ = 0.5f * (f[i] - f[o]) - 0.5f * (feq[i] - feq[o]);
            float pi = f[i] - r0 * np_ - r1 * nm_;
            float po = f[o] - r0 * np_ + r1 * nm_;
            if (FORCE) {
                const float sp = 0.5f * (S[i] + S[o]);
                const float sm = 0.5f * (S[i] - S[o]);
                pi += gp * sp + gm * sm;
                po += gp * sp - gm * sm;
            }
            f[i] = pi;
            f[o] = po;
        }
    } else {  // MRT, D2Q9 only (checked on the host)
        static_assert(L::Q == 9 || COLL != LBM_MRT, "MRT is implemented for D2Q9 only");
        const float s[9] = {0.0f, r1, r2, 0.0f, r3, 0.0f, r3, r0, r0};
        float dm[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            // conserved moments (rho, jx, jy) relax with rate 0: only the force term acts
            const bool conserved = (k == 0 || k == 3 || k == 5);
            float mne = 0.0f, ms = 0.0f;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const int m = mrt_m(k, i);
                if (m != 0) {
                    if (!conserved) mne += float(m) * (f[i] - feq[i]);
                    if (FORCE) ms += float(m) * S[i];
                }
            }
            float num;
            if (conserved) num = FORCE ? ms : 0.0f;
            else num = FORCE ? -s[k] * mne + (1.0f - 0.5f * s[k]) * ms : -s[k] * mne;
            dm[k] = num / float(mrt_norm(k));
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            float acc = f[i];
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int m = mrt_m(k, i);
                if (m != 0) acc += float(m) * dm[k];
            }
            f[i] = acc;
        }
    }
}

}  // namespace lbm
