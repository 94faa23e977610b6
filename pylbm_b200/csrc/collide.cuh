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

#include "../../include/pylbm_b200.h"
#include "f32x2.cuh"
#include "lattice.cuh"

namespace lbm {

// Ladd's lid term 6 w_i c_ix U of a population pulled from behind the moving top wall, and
// its addition / removal: explicitly rounded (never fused into an fma), so that every kernel
// applies it identically, but through intrinsics the compiler can still fold (adding a zero
// term on the planes without a lid). Its operands are never subnormal.
template <class L>
__device__ __forceinline__ float lid_term(int i, float ulid) {
    return __fmul_rn(6.0f * L::w(i) * float(L::cx(i)), ulid);
}
__device__ __forceinline__ float add_lid(float h, float lid) { return __fadd_rn(h, lid); }
__device__ __forceinline__ float sub_lid(float h, float lid) { return __fsub_rn(h, lid); }
__device__ __forceinline__ F2 add_lid(F2 h, float lid) {
    return {__fadd2_rn(h.v, make_float2(lid, lid))};
}
__device__ __forceinline__ F2 sub_lid(F2 h, float lid) {
    return {__fadd2_rn(h.v, make_float2(-lid, -lid))};
}

// Orientation of an opposite pair (i, opp(i)): the member whose first non-zero velocity
// component is positive represents the pair, so c.x of a representative never starts with a
// negation.
template <class L>
__device__ __forceinline__ constexpr bool leads_pair(int i) {
    for (int a = 0; a < L::D; ++a) {
        const int c = cc<L>(i, a);
        if (c != 0) return c > 0;
    }
    return false;
}

// Number of non-zero components of c_i, and the first of them.
template <class L>
__device__ __forceinline__ constexpr int naxes(int i) {
    int n = 0;
    for (int a = 0; a < L::D; ++a) n += cc<L>(i, a) != 0;
    return n;
}
template <class L>
__device__ __forceinline__ constexpr int first_axis(int i) {
    for (int a = 0; a < L::D; ++a)
        if (cc<L>(i, a) != 0) return a;
    return 0;
}

// c_i . x for a velocity with unit components: additions and subtractions only.
template <class L, class S>
__device__ __forceinline__ S cdot(int i, const S (&x)[3]) {
    S r = sc<S>(0.0f);
    bool started = false;
#pragma unroll
    for (int a = 0; a < L::D; ++a) {
        const int c = cc<L>(i, a);
        if (c == 0) continue;
        if (!started) r = c > 0 ? x[a] : sc<S>(0.0f) - x[a];
        else r = c > 0 ? r + x[a] : r - x[a];
        started = true;
    }
    return r;
}

// Shifted BGK / TRT on opposite pairs (i, o = opp(i), c_o = -c_i, w_o = w_i). With the pair
// sums a = h_i + h_o and differences d = h_i - h_o: drho = h_0 + sum a, j = sum_pairs c_i d,
// and the equilibrium splits into a symmetric part ep = w (drho + rho (4.5 (c.u)^2 - 1.5 u.u))
// and an antisymmetric part em = 3 w c.(rho u) (heq_i = ep + em, heq_o = ep - em); the Guo
// source likewise into S+ = w (9 (c.u)(c.F) - 3 u.F) and S- = 3 w c.F (uniform). With s+ = r0
// and s- = r1 (TRT) or r0 (BGK) the relaxation is written on a and d alone, so h_i, h_o are
// dead once a, d exist:
//   p_i = A + B, p_o = A - B,  A = (1 - s+)/2 a + s+ ep + (1 - s+/2) S+,
//                              B = (1 - s-)/2 d + s- em + (1 - s-/2) S-,
// which is h_i - s+ (a/2 - ep) - s- (d/2 - em) + ... regrouped. Same algebra as the
// per-direction form with about a third fewer operations. S is F1 (one node) or F2 (two
// nodes): the operation sequence, and so every rounding, is the same for both.
// In this and the MRT form no rounded product feeds an addition or subtraction directly
// (products enter fma_ or other products only; products by a power of two are exact and
// exempt): the code generator was measured to fuse such a pair into one fma for the packed
// instructions but not for the scalar ones, which would make the two types disagree in the
// last bit. Every F2 constant holds a register pair, so the forms also keep their number
// small (1 + x and -x are per-node scalar instructions with immediates).
// With MOM, the rho and u the collision uses are also returned (rho_out, u_out[0..D-1]).
template <class L, int COLL, bool FORCE, bool MOM = false, class S>
__device__ __forceinline__ void collide_pairs(S (&h)[L::Q], const float (&F)[3], float r0,
                                              float r1, float* rho_out = nullptr,
                                              float* u_out = nullptr) {
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    S a[Q], d[Q];
    S drho = h[0];
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        if (!leads_pair<L>(i)) continue;
        const int o = L::opp(i);
        a[i] = h[i] + h[o];
        d[i] = h[i] - h[o];
        drho = drho + a[i];
    }
    S j[3] = {sc<S>(0.0f), sc<S>(0.0f), sc<S>(0.0f)};
#pragma unroll
    for (int ax = 0; ax < D; ++ax) {
        bool started = false;
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            if (!leads_pair<L>(i)) continue;
            const int c = cc<L>(i, ax);
            if (c == 0) continue;
            if (!started) j[ax] = c > 0 ? d[i] : sc<S>(0.0f) - d[i];
            else j[ax] = c > 0 ? j[ax] + d[i] : j[ax] - d[i];
            started = true;
        }
    }
    const S rho = one_plus(drho);
    const S inv_rho = rcp_(rho);
    S ju[3], u[3];  // ju = rho u = j + F/2
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        ju[ax] = (FORCE && ax < D) ? j[ax] + sc<S>(0.5f * F[ax]) : j[ax];
        u[ax] = ax < D ? ju[ax] * inv_rho : sc<S>(0.0f);
    }
    if constexpr (MOM) {
        *rho_out = scalar_of(rho);
#pragma unroll
        for (int ax = 0; ax < D; ++ax) u_out[ax] = scalar_of(u[ax]);
    }
    S usq = u[0] * u[0];
#pragma unroll
    for (int ax = 1; ax < D; ++ax) usq = fma_(u[ax], u[ax], usq);
    const S t = sc<S>(-1.5f) * usq;
    S uf3 = sc<S>(0.0f);  // -3 u.F
    if constexpr (FORCE) {
        S uf = u[0] * sc<S>(F[0]);
#pragma unroll
        for (int ax = 1; ax < D; ++ax) uf = fma_(u[ax], sc<S>(F[ax]), uf);
        uf3 = sc<S>(-3.0f) * uf;
    }
    const float rm = COLL == LBM_TRT ? r1 : r0;
    const float gp = 1.0f - 0.5f * r0;
    const float gm = 1.0f - 0.5f * rm;
    const float kp = 0.5f * (1.0f - r0);
    const float km = 0.5f * (1.0f - rm);
    // ep / w = drho + rho t + 4.5 rho (c.u)^2 = base + 4.5 (c.rho u)(c.u)
    const S base = fma_(rho, t, drho);
    {  // rest population: heq_0 = w_0 base, S_0 = -3 w_0 u.F
        const float w0 = L::w(0);
        S p = fma_(sc<S>(1.0f - r0), h[0], sc<S>(r0 * w0) * base);
        if constexpr (FORCE) p = fma_(sc<S>(gp * w0), uf3, p);
        h[0] = p;
    }
#pragma unroll
    for (int i = 1; i < Q; ++i) {
        if (!leads_pair<L>(i)) continue;
        const int o = L::opp(i);
        const float w = L::w(i);
        const S cj = cdot<L>(i, ju);  // c.(rho u)
        // c.u: u_ax itself along an axis, else (c.j) / rho (a product, never a sum of them)
        const S cu = naxes<L>(i) == 1 ? u[first_axis<L>(i)] : cj * inv_rho;
        // s+ ep = s+ w base + 4.5 s+ w (c.rho u)(c.u); the first term is shared by the pairs
        // of one weight
        const S sep = fma_(sc<S>(4.5f * r0 * w) * cj, cu, sc<S>(r0 * w) * base);
        S A = fma_(sc<S>(kp), a[i], sep);
        S B = fma_(sc<S>(km), d[i], sc<S>(rm * 3.0f * w) * cj);
        if constexpr (FORCE) {
            float cf = 0.0f;  // c.F (uniform)
#pragma unroll
            for (int ax = 0; ax < D; ++ax) cf += float(cc<L>(i, ax)) * F[ax];
            A = fma_(sc<S>(gp), fma_(sc<S>(9.0f * w * cf), cu, sc<S>(w) * uf3), A);
            B = B + sc<S>(gm * 3.0f * w * cf);
        }
        h[i] = A + B;
        h[o] = A - B;
    }
}

// Shifted D2Q9 MRT in moment space. Moments of h (= M f - M w, M w = (1, -2, 1, 0, ...)) from
// shared partial sums; equilibrium moments of the second-order feq in closed form,
// e = -2 drho + 3 rho u.u, eps = drho - 3 rho u.u, q = -rho u, pxx = rho (ux^2 - uy^2),
// pxy = rho ux uy, with rho u = j + F/2 used directly; Guo source moments
// M S = (0, 6 u.F, -6 u.F, Fx, -Fx, Fy, -Fy, 2 (ux Fx - uy Fy), ux Fy + uy Fx); then
// h* = h + M^T (dm / |M_k|^2). Algebraically the update of lattice.py:71-109 /
// core.py:228-246 with rates (0, r1, r2, 0, r3, 0, r3, r0, r0). S is float (fp32 storages),
// F1 or F2 (16-bit storages, identical roundings; see collide_pairs for the rules kept).
template <bool FORCE, class S>
__device__ __forceinline__ void collide_mrt_moments(S (&h)[9], const float (&F)[3], float r0,
                                                    float r1, float r2, float r3) {
    const S s13 = h[1] + h[3], s24 = h[2] + h[4];
    const S s57 = h[5] + h[7], s68 = h[6] + h[8];
    const S ax_ = s13 + s24, dg_ = s57 + s68;
    const S drho = (h[0] + ax_) + dg_;
    // (-4 h0 is exact, so whether it is fused with the subtraction does not change the value)
    const S m_e = fma_(sc<S>(2.0f), dg_, sc<S>(-4.0f) * h[0] - ax_);
    const S m_eps = fma_(sc<S>(4.0f), h[0], fma_(sc<S>(-2.0f), ax_, dg_));
    const S dx = h[1] - h[3], dy = h[2] - h[4];
    const S p57 = h[5] - h[7], p86 = h[8] - h[6];
    const S q1 = p57 + p86, q2 = p57 - p86;
    const S m_qx = fma_(sc<S>(-2.0f), dx, q1);
    const S m_qy = fma_(sc<S>(-2.0f), dy, q2);
    const S m_pxx = s13 - s24;
    const S m_pxy = s57 - s68;
    const S inv_rho = rcp_(one_plus(drho));
    const S jux = FORCE ? (dx + q1) + sc<S>(0.5f * F[0]) : dx + q1;  // rho u
    const S juy = FORCE ? (dy + q2) + sc<S>(0.5f * F[1]) : dy + q2;
    const S ux = jux * inv_rho, uy = juy * inv_rho;
    const S nux = jux * neg_(inv_rho);  // -ux
    const S usq3 = sc<S>(3.0f) * fma_(jux, ux, juy * uy);  // 3 rho u.u
    // relaxed non-equilibrium moments divided by the squared row norms
    // (9, 36, 36, 6, 12, 6, 12, 4, 4); nne = -dm_e
    const float ceps = -r2 * (1.0f / 36.0f), cq = -r3 * (1.0f / 12.0f), cp = -r0 * 0.25f;
    S nne = sc<S>(r1 * (1.0f / 36.0f)) * (m_e - fma_(sc<S>(-2.0f), drho, usq3));
    S neps = fma_(sc<S>(ceps), m_eps - drho, sc<S>(ceps) * usq3);
    S nqx = fma_(sc<S>(cq), m_qx, sc<S>(cq) * jux);
    S nqy = fma_(sc<S>(cq), m_qy, sc<S>(cq) * juy);
    // pxx_eq = rho (ux^2 - uy^2) = jux ux - juy uy, pxy_eq = rho ux uy = ux juy
    S npxx = fma_(sc<S>(cp), fma_(juy, uy, m_pxx), sc<S>(cp) * (jux * nux));
    S npxy = fma_(sc<S>(cp), m_pxy, sc<S>(cp) * (nux * juy));
    S X, Y, Xd, Yd;
    if constexpr (FORCE) {
        const S uf = fma_(ux, sc<S>(F[0]), uy * sc<S>(F[1]));
        nne = fma_(sc<S>(-(1.0f - 0.5f * r1) * (6.0f / 36.0f)), uf, nne);
        neps = fma_(sc<S>(-(1.0f - 0.5f * r2) * (6.0f / 36.0f)), uf, neps);
        nqx = nqx - sc<S>((1.0f - 0.5f * r3) * (1.0f / 12.0f) * F[0]);
        nqy = nqy - sc<S>((1.0f - 0.5f * r3) * (1.0f / 12.0f) * F[1]);
        npxx = fma_(sc<S>((1.0f - 0.5f * r0) * 0.5f),
                    fma_(ux, sc<S>(F[0]), sc<S>(-F[1]) * uy), npxx);
        npxy = fma_(sc<S>((1.0f - 0.5f * r0) * 0.25f),
                    fma_(ux, sc<S>(F[1]), uy * sc<S>(F[0])), npxy);
        const float njx = F[0] * (1.0f / 6.0f), njy = F[1] * (1.0f / 6.0f);
        X = fma_(sc<S>(-2.0f), nqx, sc<S>(njx));
        Y = fma_(sc<S>(-2.0f), nqy, sc<S>(njy));
        Xd = nqx + sc<S>(njx);
        Yd = nqy + sc<S>(njy);
    } else {
        X = sc<S>(-2.0f) * nqx;  // exact
        Y = sc<S>(-2.0f) * nqy;
        Xd = nqx;
        Yd = nqy;
    }
    const S A = fma_(sc<S>(-2.0f), neps, nne);   // -dm_e - 2 dm_eps
    const S Bd = fma_(sc<S>(-2.0f), nne, neps);  // 2 dm_e + dm_eps
    // shared partial sums of the back-transform columns
    const S ax1 = A + npxx, ax2 = A - npxx;
    const S dg1 = Bd + npxy, dg2 = Bd - npxy;
    const S sd = Xd + Yd, dd = Xd - Yd;
    h[0] = fma_(sc<S>(4.0f), neps, fma_(sc<S>(4.0f), nne, h[0]));
    h[1] = h[1] + (ax1 + X);
    h[3] = h[3] + (ax1 - X);
    h[2] = h[2] + (ax2 + Y);
    h[4] = h[4] + (ax2 - Y);
    h[5] = h[5] + (dg1 + sd);
    h[7] = h[7] + (dg1 - sd);
    h[6] = h[6] + (dg2 - dd);
    h[8] = h[8] + (dg2 + dd);
}

// In: f[] pre-collision (h if SHIFT), F = total force at the node (zeros when unforced).
// Out: f[] post-collision (h* if SHIFT). MRT on shifted storages uses the moment-space form
// above (measured more accurate against float64 than the per-direction form: 9e-8 vs 1.2e-7
// on a 500-step cavity). BGK / TRT use the pair form only for COMPACT (16-bit) storages,
// whose kernels are instruction-bound and whose storage rounding dominates: in fp32 the pair
// form measured ~3x further from float64 (2.3e-6 vs 0.7e-6 after 1000 cavity steps), so fp32
// keeps the per-direction form below, which for plain storage is pylbm's order
// (lbm.cu:100-163). COMPACT collisions run in F1 arithmetic, bit-for-bit what collide2 gives
// the packed 16-bit kernels. With MOM the rho and u of the collision are also returned.
template <class L, int COLL, bool SHIFT, bool FORCE, bool COMPACT = false, bool MOM = false>
__device__ __forceinline__ void collide(float (&f)[L::Q], const float (&F)[3], float r0,
                                        float r1, float r2, float r3, float* rho_out = nullptr,
                                        float* u_out = nullptr) {
    constexpr int Q = L::Q;
    constexpr int D = L::D;
    if constexpr (COLL == LBM_STREAM_ONLY) return;  // debug mode: streaming only
    if constexpr (SHIFT && COMPACT &&
                  (COLL == LBM_BGK || COLL == LBM_TRT || (COLL == LBM_MRT && Q == 9))) {
        F1 g[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) g[i].v = f[i];
        if constexpr (COLL == LBM_MRT) {
            static_assert(!MOM, "rho / u output is implemented for BGK and TRT");
            collide_mrt_moments<FORCE>(g, F, r0, r1, r2, r3);
        } else {
            collide_pairs<L, COLL, FORCE, MOM>(g, F, r0, r1, rho_out, u_out);
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) f[i] = g[i].v;
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
    } else if constexpr (Q == 19) {
        // D3Q19 MRT in moment space (d'Humieres et al. 2002 basis, lattice.cuh). Every basis
        // row is even or odd under c -> -c, so the moments of g = f - feq (and of S) come from
        // the 9 pair sums g_i + g_opp and the 9 pair differences g_i - g_opp, and the update
        // f += M^T dm is formed once per pair as f_i += E + O, f_opp += E - O (E from the even
        // moments, O from the odd ones): half the multiply-adds of the full 19 x 19 products,
        // the same algebra.
        const float rate[4] = {r0, r1, r2, r3};
        const float g0 = f[0] - feq[0];
        float ga[Q], gd[Q], sa[Q], sd[Q];  // indexed by the pair's leading direction
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            if (!leads_pair<L>(i)) continue;
            const int o = L::opp(i);
            const float gi = f[i] - feq[i], go = f[o] - feq[o];
            ga[i] = gi + go;
            gd[i] = gi - go;
            if (FORCE) {
                sa[i] = S[i] + S[o];
                sd[i] = S[i] - S[o];
            }
        }
        float dm[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const int slot = mrt_rate_slot<L>(k);
            const bool conserved = slot < 0;
            const float sk = conserved ? 0.0f : rate[slot < 0 ? 0 : slot];
            const bool even = mrt_parity<L>(k) > 0;
            float mne = 0.0f, ms = 0.0f;
            if (even) {
                const int m0 = mrt_basis<L>(k, 0);
                if (m0 != 0) {
                    if (!conserved) mne = float(m0) * g0;
                    if (FORCE) ms = float(m0) * S[0];
                }
            }
#pragma unroll
            for (int i = 1; i < Q; ++i) {
                if (!leads_pair<L>(i)) continue;
                const int m = mrt_basis<L>(k, i);
                if (m == 0) continue;
                if (!conserved) mne += float(m) * (even ? ga[i] : gd[i]);
                if (FORCE) ms += float(m) * (even ? sa[i] : sd[i]);
            }
            float num;
            if (conserved) num = FORCE ? ms : 0.0f;
            else num = FORCE ? -sk * mne + (1.0f - 0.5f * sk) * ms : -sk * mne;
            dm[k] = num * (1.0f / float(mrt_basis_norm<L>(k)));
        }
        float e0 = 0.0f;
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            const int m0 = mrt_basis<L>(k, 0);
            if (m0 != 0) e0 += float(m0) * dm[k];
        }
        f[0] += e0;
#pragma unroll
        for (int i = 1; i < Q; ++i) {
            if (!leads_pair<L>(i)) continue;
            const int o = L::opp(i);
            float E = 0.0f, O = 0.0f;
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                const int m = mrt_basis<L>(k, i);
                if (m == 0) continue;
                if (mrt_parity<L>(k) > 0) E += float(m) * dm[k];
                else O += float(m) * dm[k];
            }
            f[i] += E + O;
            f[o] += E - O;
        }
    } else {  // D2Q9 MRT in moment space with the basis of lattice.cuh, as pylbm's kernel
        const float rate[4] = {r0, r1, r2, r3};
        float dm[Q];
#pragma unroll
        for (int k = 0; k < Q; ++k) {
            // conserved moments (rho, j) relax with rate 0: only the force term acts
            const int slot = mrt_rate_slot<L>(k);
            const bool conserved = slot < 0;
            const float sk = conserved ? 0.0f : rate[slot < 0 ? 0 : slot];
            float mne = 0.0f, ms = 0.0f;
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int m = mrt_basis<L>(k, i);
                if (m != 0) {
                    if (!conserved) mne += float(m) * (f[i] - feq[i]);
                    if (FORCE) ms += float(m) * S[i];
                }
            }
            float num;
            if (conserved) num = FORCE ? ms : 0.0f;
            else num = FORCE ? -sk * mne + (1.0f - 0.5f * sk) * ms : -sk * mne;
            dm[k] = num / float(mrt_basis_norm<L>(k));  // a division, as pylbm's kernel
        }
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            float acc = f[i];
#pragma unroll
            for (int k = 0; k < Q; ++k) {
                const int m = mrt_basis<L>(k, i);
                if (m != 0) acc += float(m) * dm[k];
            }
            f[i] = acc;
        }
    }
}

}  // namespace lbm

namespace lbm {

// Two nodes of a 16-bit storage word at once (packed fp32 pairs, shifted arithmetic):
// bit-for-bit collide<L, COLL, true, FORCE, true> applied to each node.
template <class L, int COLL, bool FORCE>
__device__ __forceinline__ void collide2(F2 (&f)[L::Q], const float (&F)[3], float r0,
                                         float r1, float r2, float r3) {
    if constexpr (COLL == LBM_STREAM_ONLY) {
        return;
    } else if constexpr (COLL == LBM_MRT) {
        static_assert(L::Q == 9, "MRT is implemented for D2Q9 only");
        collide_mrt_moments<FORCE>(f, F, r0, r1, r2, r3);
    } else {
        collide_pairs<L, COLL, FORCE>(f, F, r0, r1);
    }
}

}  // namespace lbm
