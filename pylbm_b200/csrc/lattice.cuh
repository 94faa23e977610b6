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

}  // namespace lbm
