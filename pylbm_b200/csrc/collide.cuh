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

// Correctly rounded 1/x (the value of the IEEE quotient 1.0f / x) for the shifted
// collisions. Measured against an approximate reciprocal with one Newton step, it is as fast
// or faster in every kernel and keeps the reciprocal exact.
__device__ __forceinline__ float fast_rcp(float x) { return __frcp_rn(x); }

// Shifted BGK / TRT on opposite pairs (i, o = opp(i), c_o = -c_i, w_o = w_i). With the pair
// sums a = h_i + h_o and differences d = h_i - h_o: drho = h_0 + sum a, j = sum_pairs c_i d,
// and the equilibrium splits into a symmetric part ep = w (drho + rho (4.5 (c.u)^2 - 1.5 u.u))
// and an antisymmetric part em = 3 w rho c.u (heq_i = ep + em, heq_o = ep - em); the Guo
// source likewise into S+ = w (9 (c.u)(c.F) - 3 u.F) and S- = 3 w c.F. TRT relaxes the two
// parts with s+ = r0 and s- = r1 directly; BGK relaxes heq_i, heq_o with r0. Same algebra as
// the per-direction form with about a third fewer instructions: the 16-bit kernels, whose
// bandwidth needs twice the node rate of fp32, are bound by instruction issue, not HBM.
// With MOM, the rho and u the collision uses are also returned (rho_out, u_out[0..D-1]).
template <class L, int COLL, bool FORCE, bool MOM = false>
__device__ __forceinline__ void collide_pairs(float (&h)[L::Q], const float (&F)[3], float r0,
                                              float r1, float* rho_out = nullptr,
                                              float* u_out = nullptr) {
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    float a[Q], d[Q];
    float drho = h[0];
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        a[i] = h[i] + h[o];
        d[i] = h[i] - h[o];
        drho += a[i];
    }
    float j[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int ax = 0; ax < D; ++ax) {
        bool started = false;
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            if (L::opp(i) < i) continue;
            const int c = cc<L>(i, ax);
            if (c == 0) continue;
            if (!started) {
                j[ax] = c > 0 ? d[i] : -d[i];
                started = true;
            } else {
                j[ax] = c > 0 ? j[ax] + d[i] : j[ax] - d[i];
            }
        }
    }
    const float rho = 1.0f + drho;
    const float inv_rho = fast_rcp(rho);
    float u[3];
#pragma unroll
    for (int ax = 0; ax < D; ++ax) u[ax] = (FORCE ? j[ax] + 0.5f * F[ax] : j[ax]) * inv_rho;
    if constexpr (MOM) {
        *rho_out = rho;
#pragma unroll
        for (int ax = 0; ax < D; ++ax) u_out[ax] = u[ax];
    }
    float usq = u[0] * u[0];
#pragma unroll
    for (int ax = 1; ax < D; ++ax) usq += u[ax] * u[ax];
    const float t = -1.5f * usq;
    float uf = 0.0f;
    if (FORCE) {
        uf = u[0] * F[0];
#pragma unroll
        for (int ax = 1; ax < D; ++ax) uf += u[ax] * F[ax];
    }
    const float gp = 1.0f - 0.5f * r0;
    const float gm = 1.0f - 0.5f * (COLL == LBM_TRT ? r1 : r0);
    {  // rest population
        const float w0 = L::w(0);
        const float heq = w0 * drho + (w0 * rho) * t;
        float p = h[0] + r0 * (heq - h[0]);
        if (FORCE) p += gp * (w0 * (-3.0f * uf));
        h[0] = p;
    }
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        const int o = L::opp(i);
        if (o < i) continue;
        const float w = L::w(i);
        float cu = 0.0f, cf = 0.0f;
#pragma unroll
        for (int ax = 0; ax < D; ++ax) {
            const int c = cc<L>(i, ax);
            if (c == 1) {
                cu += u[ax];
                if (FORCE) cf += F[ax];
            }
            if (c == -1) {
                cu -= u[ax];
                if (FORCE) cf -= F[ax];
            }
        }
        const float ep = (w * drho) + (w * rho) * fmaf(4.5f * cu, cu, t);
        const float em = (3.0f * w * rho) * cu;
        float sp = 0.0f, sm = 0.0f;
        if (FORCE) {
            sp = w * (9.0f * cu * cf - 3.0f * uf);
            sm = 3.0f * w * cf;
        }
        float pi, po;
        if (COLL == LBM_TRT) {
            const float np_ = 0.5f * a[i] - ep;
            const float nm_ = 0.5f * d[i] - em;
            pi = h[i] - r0 * np_ - r1 * nm_;
            po = h[o] - r0 * np_ + r1 * nm_;
            if (FORCE) {
                pi += gp * sp + gm * sm;
                po += gp * sp - gm * sm;
            }
        } else {
            pi = h[i] + r0 * ((ep + em) - h[i]);
            po = h[o] + r0 * ((ep - em) - h[o]);
            if (FORCE) {
                pi += gp * (sp + sm);
                po += gp * (sp - sm);
            }
        }
        h[i] = pi;
        h[o] = po;
    }
}

// Shifted D2Q9 MRT in moment space. Moments of h (= M f - M w, M w = (1, -2, 1, 0, ...)) from
// shared partial sums; equilibrium moments of the second-order feq in closed form,
// e = -2 drho + 3 rho u.u, eps = drho - 3 rho u.u, q = -rho u, pxx = rho (ux^2 - uy^2),
// pxy = rho ux uy; Guo source moments M S = (0, 6 u.F, -6 u.F, Fx, -Fx, Fy, -Fy,
// 2 (ux Fx - uy Fy), ux Fy + uy Fx); then h* = h + M^T (dm / |M_k|^2). Algebraically the
// update of lattice.py:71-109 / core.py:228-246 with rates (0, r1, r2, 0, r3, 0, r3, r0, r0).
template <bool FORCE>
__device__ __forceinline__ void collide_mrt_moments(float (&h)[9], const float (&F)[3],
                                                    float r0, float r1, float r2, float r3) {
    const float ax_ = (h[1] + h[3]) + (h[2] + h[4]);
    const float dg_ = (h[5] + h[7]) + (h[6] + h[8]);
    const float drho = h[0] + ax_ + dg_;
    const float m_e = -4.0f * h[0] - ax_ + 2.0f * dg_;
    const float m_eps = 4.0f * h[0] - 2.0f * ax_ + dg_;
    const float dx = h[1] - h[3], dy = h[2] - h[4];
    const float p57 = h[5] - h[7], p86 = h[8] - h[6];
    const float jx = dx + (p57 + p86), jy = dy + (p57 - p86);
    const float m_qx = -2.0f * dx + (p57 + p86);
    const float m_qy = -2.0f * dy + (p57 - p86);
    const float m_pxx = (h[1] + h[3]) - (h[2] + h[4]);
    const float m_pxy = (h[5] + h[7]) - (h[6] + h[8]);
    const float rho = 1.0f + drho;
    const float inv_rho = fast_rcp(rho);
    const float ux = (FORCE ? jx + 0.5f * F[0] : jx) * inv_rho;
    const float uy = (FORCE ? jy + 0.5f * F[1] : jy) * inv_rho;
    const float uxx = ux * ux, uyy = uy * uy;
    const float usq3 = 3.0f * rho * (uxx + uyy);
    // relaxed non-equilibrium moments, already divided by the squared row norms
    // (9, 36, 36, 6, 12, 6, 12, 4, 4): the rates are scaled once, not every moment
    float ne = (-r1 * (1.0f / 36.0f)) * (m_e - (-2.0f * drho + usq3));
    float neps = (-r2 * (1.0f / 36.0f)) * (m_eps - (drho - usq3));
    float nqx = (-r3 * (1.0f / 12.0f)) * (m_qx + rho * ux);
    float nqy = (-r3 * (1.0f / 12.0f)) * (m_qy + rho * uy);
    float npxx = (-r0 * 0.25f) * (m_pxx - rho * (uxx - uyy));
    float npxy = (-r0 * 0.25f) * (m_pxy - rho * ux * uy);
    float njx = 0.0f, njy = 0.0f;
    if (FORCE) {
        const float uf = ux * F[0] + uy * F[1];
        ne += ((1.0f - 0.5f * r1) * (6.0f / 36.0f)) * uf;
        neps -= ((1.0f - 0.5f * r2) * (6.0f / 36.0f)) * uf;
        nqx -= ((1.0f - 0.5f * r3) * (1.0f / 12.0f)) * F[0];
        nqy -= ((1.0f - 0.5f * r3) * (1.0f / 12.0f)) * F[1];
        npxx += ((1.0f - 0.5f * r0) * 0.5f) * (ux * F[0] - uy * F[1]);
        npxy += ((1.0f - 0.5f * r0) * 0.25f) * (ux * F[1] + uy * F[0]);
        njx = F[0] * (1.0f / 6.0f);
        njy = F[1] * (1.0f / 6.0f);
    }
    const float A = -ne - 2.0f * neps;
    const float Bd = 2.0f * ne + neps;
    const float X = njx - 2.0f * nqx, Y = njy - 2.0f * nqy;
    const float Xd = njx + nqx, Yd = njy + nqy;
    // shared partial sums of the back-transform columns
    const float ax1 = A + npxx, ax2 = A - npxx;
    const float dg1 = Bd + npxy, dg2 = Bd - npxy;
    const float sd = Xd + Yd, dd = Xd - Yd;
    h[0] += 4.0f * (neps - ne);
    h[1] += ax1 + X;
    h[3] += ax1 - X;
    h[2] += ax2 + Y;
    h[4] += ax2 - Y;
    h[5] += dg1 + sd;
    h[7] += dg1 - sd;
    h[6] += dg2 - dd;
    h[8] += dg2 + dd;
}

// In: f[] pre-collision (h if SHIFT), F = total force at the node (zeros when unforced).
// Out: f[] post-collision (h* if SHIFT). MRT on shifted storages uses the moment-space form
// above (measured more accurate against float64 than the per-direction form: 9e-8 vs 1.2e-7
// on a 500-step cavity). BGK / TRT use the pair form only for COMPACT (16-bit) storages,
// whose kernels are instruction-bound and whose storage rounding dominates: in fp32 the pair
// form measured ~3x further from float64 (2.3e-6 vs 0.7e-6 after 1000 cavity steps), so fp32
// keeps the per-direction form below, which for plain storage is pylbm's order
// (lbm.cu:100-163). With MOM the rho and u of the collision are also returned.
template <class L, int COLL, bool SHIFT, bool FORCE, bool COMPACT = false, bool MOM = false>
__device__ __forceinline__ void collide(float (&f)[L::Q], const float (&F)[3], float r0,
                                        float r1, float r2, float r3, float* rho_out = nullptr,
                                        float* u_out = nullptr) {
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    if constexpr (COLL == LBM_STREAM_ONLY) return;  // debug mode: streaming only
    if constexpr (SHIFT && COMPACT && (COLL == LBM_BGK || COLL == LBM_TRT)) {
        collide_pairs<L, COLL, FORCE, MOM>(f, F, r0, r1, rho_out, u_out);
        return;
    }
    if constexpr (SHIFT && COLL == LBM_MRT && Q == 9) {
        collide_mrt_moments<FORCE>(f, F, r0, r1, r2, r3);
        return;
    }
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
    if constexpr (MOM) {
        *rho_out = rho;
#pragma unroll
        for (int a = 0; a < D; ++a) u_out[a] = u[a];
    }
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
