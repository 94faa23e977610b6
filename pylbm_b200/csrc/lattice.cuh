// Lattice descriptors as compile-time traits.
//
// The velocity orders, weights and opposite tables must match pylbm's (lattice.py:49-67):
// population i of a buffer written by pylbm is population i here. They are written as
// constexpr functions so that, inside fully unrolled loops, every c_i, w_i and opp(i) folds
// into an immediate and no lattice table lives in memory.
#pragma once

#include <cstdint>

namespace lbm {

struct D2Q9 {
    static constexpr int Q = 9;
    static constexpr int D = 2;
    // 0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE  (lattice.py:49-54)
    __host__ __device__ static constexpr int cx(int i) {
        return (i == 1 || i == 5 || i == 8) ? 1 : (i == 3 || i == 6 || i == 7) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cy(int i) {
        return (i == 2 || i == 5 || i == 6) ? 1 : (i == 4 || i == 7 || i == 8) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cz(int) { return 0; }
    __host__ __device__ static constexpr float w(int i) {
        return i == 0 ? 4.0f / 9.0f : (i < 5 ? 1.0f / 9.0f : 1.0f / 36.0f);
    }
    __host__ __device__ static constexpr double wd(int i) {
        return i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
    __host__ __device__ static constexpr int opp(int i) {
        return i == 0 ? 0 : (i < 5 ? ((i + 1) & 3) + 1 : ((i - 3) & 3) + 5);
    }
};

struct D3Q19 {
    static constexpr int Q = 19;
    static constexpr int D = 3;
    // 0 rest; (1,2) +-x; (3,4) +-y; (5,6) +-z; (7..10) xy; (11..14) xz; (15..18) yz
    // (lattice.py:56-67)
    __host__ __device__ static constexpr int cx(int i) {
        return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1
             : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cy(int i) {
        return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1
             : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
    }
    __host__ __device__ static constexpr int cz(int i) {
        return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1
             : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
    }
    __host__ __device__ static constexpr float w(int i) {
        return i == 0 ? 1.0f / 3.0f : (i < 7 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
    __host__ __device__ static constexpr double wd(int i) {
        return i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
    __host__ __device__ static constexpr int opp(int i) {
        return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1);
    }
};

// Component a of c_i.
template <class L>
__host__ __device__ constexpr int cc(int i, int a) {
    return a == 0 ? L::cx(i) : (a == 1 ? L::cy(i) : L::cz(i));
}

// Lallemand-Luo (2000) D2Q9 moment basis in the velocity order above; rows are
// (rho, e, eps, jx, qx, jy, qy, pxx, pxy). This is the table of lattice.py:71-87, which the
// MRT collision must use unchanged for its rates to mean the same moments.
__host__ __device__ constexpr int mrt_m(int k, int i) {
    constexpr int8_t M[9][9] = {
        {1, 1, 1, 1, 1, 1, 1, 1, 1},
        {-4, -1, -1, -1, -1, 2, 2, 2, 2},
        {4, -2, -2, -2, -2, 1, 1, 1, 1},
        {0, 1, 0, -1, 0, 1, -1, -1, 1},
        {0, -2, 0, 2, 0, 1, -1, -1, 1},
        {0, 0, 1, 0, -1, 1, 1, -1, -1},
        {0, 0, -2, 0, 2, 1, 1, -1, -1},
        {0, 1, -1, 1, -1, 0, 0, 0, 0},
        {0, 0, 0, 0, 0, 1, -1, 1, -1},
    };
    return M[k][i];
}
// Squared row norms: M is orthogonal, M^-1 = M^T diag(1 / norm)  (lattice.py:88)
__host__ __device__ constexpr int mrt_norm(int k) {
    constexpr int8_t NRM[9] = {9, 36, 36, 6, 12, 6, 12, 4, 4};
    return NRM[k];
}

// D3Q19 moment basis of d'Humieres et al. (2002), orthogonal, as polynomials of c_i in the
// velocity order above; rows (rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww,
// pxy, pyz, pxz, mx, my, mz). pylbm has no D3Q19 MRT; the rates follow its D2Q9 convention
// (mrt_rates below).
__host__ __device__ constexpr int mrt3_poly(int k, int x, int y, int z) {
    const int c2 = x * x + y * y + z * z;
    switch (k) {
        case 0: return 1;
        case 1: return 19 * c2 - 30;
        case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
        case 3: return x;
        case 4: return (5 * c2 - 9) * x;
        case 5: return y;
        case 6: return (5 * c2 - 9) * y;
        case 7: return z;
        case 8: return (5 * c2 - 9) * z;
        case 9: return 3 * x * x - c2;
        case 10: return (3 * c2 - 5) * (3 * x * x - c2);
        case 11: return y * y - z * z;
        case 12: return (3 * c2 - 5) * (y * y - z * z);
        case 13: return x * y;
        case 14: return y * z;
        case 15: return x * z;
        case 16: return (y * y - z * z) * x;
        case 17: return (z * z - x * x) * y;
        default: return (x * x - y * y) * z;
    }
}
struct Mrt3Table {
    int8_t m[19][19];
    int16_t norm[19];
    int8_t parity[19];  // +1: M[k][opp(i)] = M[k][i] for all i; -1: = -M[k][i]; 0: neither
};
// The table, evaluated by the compiler: inside unrolled loops every entry is an immediate.
__host__ __device__ constexpr Mrt3Table make_mrt3() {
    Mrt3Table t{};
    for (int k = 0; k < 19; ++k) {
        int n = 0;
        for (int i = 0; i < 19; ++i) {
            const int v = mrt3_poly(k, D3Q19::cx(i), D3Q19::cy(i), D3Q19::cz(i));
            t.m[k][i] = static_cast<int8_t>(v);
            n += v * v;
        }
        t.norm[k] = static_cast<int16_t>(n);
    }
    for (int k = 0; k < 19; ++k) {
        bool even = true, odd = true;
        for (int i = 0; i < 19; ++i) {
            even = even && t.m[k][i] == t.m[k][D3Q19::opp(i)];
            odd = odd && t.m[k][i] == -t.m[k][D3Q19::opp(i)];
        }
        t.parity[k] = static_cast<int8_t>(even ? 1 : (odd ? -1 : 0));
    }
    return t;
}
__host__ __device__ constexpr int mrt3_m(int k, int i) {
    constexpr Mrt3Table T = make_mrt3();
    return T.m[k][i];
}
__host__ __device__ constexpr int mrt3_norm(int k) {
    constexpr Mrt3Table T = make_mrt3();
    return T.norm[k];
}
__host__ __device__ constexpr int mrt3_parity(int k) {
    constexpr Mrt3Table T = make_mrt3();
    return T.parity[k];
}
static_assert(make_mrt3().norm[1] == 2394 && make_mrt3().norm[2] == 252 &&
                  make_mrt3().norm[10] == 72 && make_mrt3().norm[18] == 8,
              "d'Humieres et al. (2002) row norms");

// The MRT basis, its squared row norms and the moments it conserves, for either lattice.
template <class L>
__host__ __device__ constexpr int mrt_basis(int k, int i) {
    if constexpr (L::Q == 9) return mrt_m(k, i);
    else return mrt3_m(k, i);
}
template <class L>
__host__ __device__ constexpr int mrt_basis_norm(int k) {
    if constexpr (L::Q == 9) return mrt_norm(k);
    else return mrt3_norm(k);
}
template <class L>
__host__ __device__ constexpr bool mrt_conserved(int k) {
    return L::Q == 9 ? (k == 0 || k == 3 || k == 5) : (k == 0 || k == 3 || k == 5 || k == 7);
}
// Parity of basis row k under c -> -c: +1 when M[k][opp(i)] = M[k][i] for every i (even
// moments: they see only the pair sums f_i + f_opp(i)), -1 when M[k][opp(i)] = -M[k][i] (odd
// moments: pair differences), 0 for a row that is neither. D3Q19 reads it from the table the
// compiler evaluates (a loop here, left to the optimiser inside unrolled code, kept the table
// in local memory).
template <class L>
__host__ __device__ constexpr int mrt_parity(int k) {
    if constexpr (L::Q == 19) {
        return mrt3_parity(k);
    } else {
        bool even = true, odd = true;
        for (int i = 0; i < L::Q; ++i) {
            const int a = mrt_basis<L>(k, i), b = mrt_basis<L>(k, L::opp(i));
            even = even && a == b;
            odd = odd && a == -b;
        }
        return even ? 1 : (odd ? -1 : 0);
    }
}
template <class L>
__host__ __device__ constexpr bool mrt_rows_have_parity() {
    for (int k = 0; k < L::Q; ++k)
        if (mrt_parity<L>(k) == 0) return false;
    return true;
}
static_assert(mrt_rows_have_parity<D3Q19>(), "every D3Q19 basis row is even or odd");

// Rate of moment k from the descriptor's (r0, r1, r2, r3) = (s_nu, s_e, s_eps, s_q):
// D2Q9 (0, s_e, s_eps, 0, s_q, 0, s_q, s_nu, s_nu) as pylbm (problem.py:102-106); D3Q19: e ->
// s_e, eps and the fourth-order pi moments -> s_eps, the energy fluxes q and the third-order
// m moments -> s_q, the five shear moments -> s_nu.
template <class L>
__host__ __device__ constexpr int mrt_rate_slot(int k) {  // 0..3 = r0..r3, -1 = conserved
    if (mrt_conserved<L>(k)) return -1;
    if constexpr (L::Q == 9) {
        return k == 1 ? 1 : k == 2 ? 2 : (k == 4 || k == 6) ? 3 : 0;
    } else {
        return k == 1 ? 1 : (k == 2 || k == 10 || k == 12) ? 2
             : (k == 4 || k == 6 || k == 8 || k >= 16) ? 3 : 0;
    }
}

}  // namespace lbm
