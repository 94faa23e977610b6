// Vectorised D2Q9 kernels: every lane owns V consecutive nodes of one row (V = 4 fp32 or
// 8 x 16-bit, one 16-byte vector per population plane).
//
// Pull (AB and the read half of AA-odd): the row segment of plane i is read at row y - c_iy
// with one aligned 16-byte load; the x-shift by c_ix moves elements inside the vector and
// takes the element across the lane boundary from the neighbouring lane with one warp
// shuffle. Only the first and last lane of a warp read one more element (the warp's halo) with
// a scalar load that the neighbouring warp's line already brought into L2; warps are
// otherwise independent (no shared memory, no block barrier). x walls and the periodic x wrap
// are resolved inside that halo element. Rows of fewer than 128 lanes run a second form of the
// kernels (SEG) with several rows per block: a row of fewer than 32 lanes takes a power-of-two
// segment of a warp (32 / w rows per warp, shuffles of width w), and a segment that holds a
// whole periodic row rotates its shifts within itself (no halo loads, no partial stores).
// Longer rows keep one row per block (see lane_of).
//
// Rows next to a y wall (y = 0 and y = ny - 1 of a non-periodic y axis) take a separate,
// general code path (the whole segment bounces back from the node's own opposite plane, plus
// the lid term on the top wall); every other row runs a path with no wall or lid code at all.
// The branch is uniform per warp, and keeping the wall logic out of the hot path keeps its
// nine loads in flight together (measured: the fused variant ran 20% slower otherwise).
//
// AA-odd push: the write of p_i(x) to x + c_i is an aligned vector store of the segment
// shifted by one element, except at warp edges. The AA scheme is race-free because every
// memory slot is read and written by one node only (slot (i, x + c_i) belongs to node x); so
// a lane stores an aligned vector only when all of its elements belong to nodes of its own
// warp, and the first / last lane stores the V - 1 slots of its own nodes in three aligned
// pieces (st_tail / st_head in vec.cuh).
//
// Semantics are those of the generic kernel (step_generic.cuh) and of pylbm's fused kernel
// (lbm.cu:71-198, codegen.py:10-16); the collision is the shared collide<>().
#include "codec.cuh"
#include "collide.cuh"
#include "dispatch.cuh"
#include "lattice.cuh"
#include "params.cuh"
#include "staged_launch.cuh"
#include "vec.cuh"

namespace lbm {
namespace {

using L = D2Q9;
constexpr int kThreads = 128;
constexpr unsigned kFull = 0xffffffffu;

// Row y - cy, wrapped. EDGE rows also report whether the row lies behind a wall (then it is
// not wrapped) and whether that wall is the top one.
template <bool EDGE>
__device__ __forceinline__ int src_row(int y, int cy, int ny, bool per, bool& wall, bool& top) {
    int ys = y - cy;
    wall = top = false;
    if constexpr (!EDGE) {
        ys += ys < 0 ? ny : (ys >= ny ? -ny : 0);
    } else if (ys < 0 || ys >= ny) {
        if (per) {
            ys += ys < 0 ? ny : -ny;
        } else {
            wall = true;
            top = ys >= ny;
        }
    }
    return ys;
}

// The lane's place: V consecutive nodes x0.. of row y. w: lanes of a row segment (32, or the
// power of two a row of fewer than 32 lanes is given, SEG only); sl: the lane's index in it;
// rot: the segment holds one whole periodic row (nx = w V), so the x neighbours across the
// row's ends are its last and first lanes (SEG only). Batches use the whole-warp form.
struct Lane {
    int x0, y, sl, w;
    bool active, first, last, rot;
};

// SEG: blocks of several rows (rows of fewer than 128 lanes), shaped by block_for_rows; else
// one row per block (1-D blocks, row = blockIdx.y, which keeps the row arithmetic uniform
// across the warp: computed from threadIdx.y it measured 5-7 % slower at 4096^2).
template <int STORE, bool SEG>
__device__ __forceinline__ Lane lane_of(const StepParams& P) {
    constexpr int V = VT<STORE>::V;
    Lane l;
    l.x0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    if constexpr (SEG) {
        l.w = blockDim.x < 32 ? int(blockDim.x) : 32;
        l.sl = threadIdx.x & (l.w - 1);
        l.y = blockIdx.y * blockDim.y + threadIdx.y;
        l.active = l.x0 < P.n[0] && l.y < P.n[1];
        l.rot = P.per[0] && P.n[0] == l.w * V;
    } else {
        l.w = 32;
        l.sl = threadIdx.x & 31;
        l.y = blockIdx.y;
        l.active = l.x0 < P.n[0];
        l.rot = false;
    }
    l.first = l.sl == 0;
    l.last = l.active && (l.sl == l.w - 1 || l.x0 + V >= P.n[0]);
    return l;
}

// The value of lane sl - 1 / sl + 1: cyclically within the segment (SEG), else the plain warp
// shuffle (the first / last lane's own value, which its halo replaces).
template <bool SEG>
__device__ __forceinline__ uint32_t from_prev(const Lane& l, uint32_t x) {
    if constexpr (SEG) return __shfl_sync(kFull, x, (l.sl + l.w - 1) & (l.w - 1), l.w);
    else return __shfl_up_sync(kFull, x, 1);
}
template <bool SEG>
__device__ __forceinline__ uint32_t from_next(const Lane& l, uint32_t x) {
    if constexpr (SEG) return __shfl_sync(kFull, x, (l.sl + 1) & (l.w - 1), l.w);
    else return __shfl_down_sync(kFull, x, 1);
}

// Block shape (lanes along x, rows) for rows of nx nodes: whole warps for rows of 32 lanes or
// more, power-of-two segments of a warp for shorter rows (the SEG kernels).
inline dim3 block_for_rows(int nx, int V) {
    const int need = (nx + V - 1) / V;
    if (need < 32) {
        int w = 1;
        while (w < need) w <<= 1;
        return dim3(w, kThreads / w);
    }
    int lanes = (need + 31) / 32 * 32;
    if (lanes > kThreads) lanes = kThreads;
    return dim3(lanes, kThreads / lanes);
}

// Load the pulled row segments of all 9 directions into v[] (raw storage elements), already
// shifted along x. READ_OPP selects the AA-odd reading (source slot opp(i), bounce-back slot
// i) instead of the two-buffer one (source slot i, bounce-back slot opp(i)).
template <int STORE, bool READ_OPP, bool NC, bool EDGE, bool SEG = false>
__device__ __forceinline__ void pull_rows(const StepParams& P, const typename VT<STORE>::E* A,
                                          const Lane& l, uint4 (&v)[9], float (&lid)[9]) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    const int nx = P.n[0], ny = P.n[1], N = P.N;
    const int x0 = l.x0, y = l.y;
    const bool active = l.active;
    const bool first = l.first && !l.rot, last = l.last && !l.rot;  // lanes that take a halo
    const bool perx = P.per[0], pery = P.per[1];
    uint32_t halo[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int cx = L::cx(i), cy = L::cy(i);
        const int src_slot = READ_OPP ? L::opp(i) : i;
        const int bb_slot = READ_OPP ? i : L::opp(i);
        bool wall, top;
        const int ys = src_row<EDGE>(y, cy, ny, pery, wall, top);
        lid[i] = (wall && top && cx != 0) ? lid_term<L>(i, P.ulid) : 0.0f;
        v[i] = make_uint4(0u, 0u, 0u, 0u);
        halo[i] = 0u;
        if (!active) continue;
        if (wall) {  // the whole segment bounces back from the node's own opposite slot
            const E* p = A + bb_slot * N + y * nx + x0;
            v[i] = NC ? ld_nc(p) : ld_plain(p);
            continue;
        }
        const E* row = A + src_slot * N + ys * nx;
        v[i] = NC ? ld_nc(row + x0) : ld_plain(row + x0);
        if (cx == 1 && first) {
            const E* h = x0 > 0 ? row + x0 - 1
                                : (perx ? row + nx - 1 : A + bb_slot * N + y * nx);
            halo[i] = NC ? ld1_nc(h) : ld1(h);
        }
        if (cx == -1 && last) {
            const E* h = x0 + V < nx ? row + x0 + V
                                     : (perx ? row : A + bb_slot * N + y * nx + nx - 1);
            halo[i] = NC ? ld1_nc(h) : ld1(h);
        }
    }
    // x-shifts: element k of node x0 + k comes from x0 + k - cx
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int cx = L::cx(i);
        if (cx == 0) continue;
        bool wall, top;
        src_row<EDGE>(y, L::cy(i), ny, pery, wall, top);
        if (cx == 1) {
            uint32_t up = from_prev<SEG>(l, elem<V>(v[i], V - 1));
            if (first) up = halo[i];
            if (!wall) v[i] = shift_up<V>(v[i], up);
        } else {
            uint32_t dn = from_next<SEG>(l, elem<V>(v[i], 0));
            if (last) dn = halo[i];
            if (!wall) v[i] = shift_down<V>(v[i], dn);
        }
    }
}

// Collide the V nodes of the lane in place (raw elements in, raw elements out). With LIDS,
// lid[i] is added to the pulled value of direction i and sub[i] is subtracted from its
// post-collision value before it is stored (the AA-odd push into the lid). 16-bit storages:
// PACK collides the two nodes of a word together with packed f32x2 instructions (F2), else
// one after the other (F1); the results are identical, the speed is not: packing halves the
// collision's instructions but keeps both nodes' populations live at once. Measured at 4096^2
// (MLUPS, F2 / F1): AB BGK 177 / 174, AB TRT 174 / 174, AB MRT 161 / 164, AA BGK 156 / 161.
template <int STORE, int COLL, bool FORCE, bool LIDS, bool PACK>
__device__ __forceinline__ void collide_lane(const StepParams& P, uint4 (&v)[9],
                                             const float (&lid)[9], const float (&sub)[9]) {
    using T = VT<STORE>;
    constexpr int V = T::V;
    constexpr bool SHIFT = Codec<STORE>::shifted;
    const float F[3] = {P.F[0], P.F[1], 0.0f};
    if constexpr (V == 4) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            float f[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                f[i] = T::f(elem<V>(v[i], k));
                if (LIDS) f[i] = add_lid(f[i], lid[i]);
            }
            collide<L, COLL, SHIFT, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 9; ++i)
                put<V>(v[i], k, T::b(LIDS ? sub_lid(f[i], sub[i]) : f[i]));
        }
    } else if constexpr (!PACK) {  // 16-bit, one node after the other
#pragma unroll
        for (int jw = 0; jw < 4; ++jw) {
            float f0[9], f1[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const float2 p = unpack2<STORE>(word(v[i], jw));
                f0[i] = LIDS ? add_lid(p.x, lid[i]) : p.x;
                f1[i] = LIDS ? add_lid(p.y, lid[i]) : p.y;
            }
            collide<L, COLL, true, FORCE, true>(f0, F, P.r0, P.r1, P.r2, P.r3);
            collide<L, COLL, true, FORCE, true>(f1, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 9; ++i)
                set_word(v[i], jw, LIDS ? pack2<STORE>(sub_lid(f0[i], sub[i]),
                                                       sub_lid(f1[i], sub[i]))
                                        : pack2<STORE>(f0[i], f1[i]));
        }
    } else {  // 16-bit: the two nodes of a word at once, packed conversions and arithmetic
#pragma unroll
        for (int jw = 0; jw < 4; ++jw) {
            F2 f[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                f[i].v = unpack2<STORE>(word(v[i], jw));
                if (LIDS) f[i] = add_lid(f[i], lid[i]);
            }
            collide2<L, COLL, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                if (LIDS) f[i] = sub_lid(f[i], sub[i]);
                set_word(v[i], jw, pack2<STORE>(f[i].v.x, f[i].v.y));
            }
        }
    }
}

// A row next to a y wall (only those carry wall and lid logic).
__device__ __forceinline__ bool edge_row(const StepParams& P, int y) {
    return !P.per[1] && (y == 0 || y == P.n[1] - 1);
}
// Whether the warp takes the wall path: any of its rows is next to a y wall (all 32 lanes
// call this, before any of them can leave).
template <bool SEG>
__device__ __forceinline__ bool edge_warp(const StepParams& P, const Lane& l) {
    const bool e = edge_row(P, l.y);
    if constexpr (SEG) return l.w < 32 ? __any_sync(kFull, e) : e;
    else return e;
}

template <int STORE, int COLL, bool FORCE, bool EDGE, bool PACK = (COLL != LBM_MRT),
          bool SEG = false>
__device__ __forceinline__ void ab_row(const StepParams& P, const typename VT<STORE>::E* A,
                                       typename VT<STORE>::E* B, const Lane& l) {
    uint4 v[9];
    float lid[9];
    pull_rows<STORE, false, true, EDGE, SEG>(P, A, l, v, lid);
    if (!l.active) return;
    const float zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    collide_lane<STORE, COLL, FORCE, EDGE, PACK>(P, v, lid, zero);
    const int n0 = l.y * P.n[0] + l.x0;
#pragma unroll
    for (int i = 0; i < 9; ++i) st_cs(B + i * P.N + n0, v[i]);
}

template <int STORE, int COLL, bool FORCE, bool SEG>
__global__ void __launch_bounds__(kThreads)
k_d2q9_ab(const StepParams P, const void* __restrict__ Av, void* __restrict__ Bv) {
    using E = typename VT<STORE>::E;
    const E* __restrict__ A = static_cast<const E*>(Av);
    E* __restrict__ B = static_cast<E*>(Bv);
    constexpr bool pack = COLL != LBM_MRT;
    const Lane l = lane_of<STORE, SEG>(P);
    if (edge_warp<SEG>(P, l)) ab_row<STORE, COLL, FORCE, true, pack, SEG>(P, A, B, l);
    else ab_row<STORE, COLL, FORCE, false, pack, SEG>(P, A, B, l);
}

template <int STORE, int COLL, bool FORCE>
__global__ void __launch_bounds__(kThreads)
k_d2q9_aa_even(const StepParams P, void* Av) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    E* A = static_cast<E*>(Av);
    const int n0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    if (n0 >= P.N) return;
    uint4 v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = ld_plain(A + i * P.N + n0);
    const float zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    collide_lane<STORE, COLL, FORCE, false, false>(P, v, zero, zero);
#pragma unroll
    for (int i = 0; i < 9; ++i) st_cs(A + L::opp(i) * P.N + n0, v[i]);
}

template <int STORE, int COLL, bool FORCE, bool EDGE, bool SEG>
__device__ __forceinline__ void aa_odd_row(const StepParams& P, typename VT<STORE>::E* A,
                                           const Lane& l) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    const int nx = P.n[0], ny = P.n[1], N = P.N;
    uint4 v[9];
    float lid[9];
    pull_rows<STORE, true, false, EDGE, SEG>(P, A, l, v, lid);
    // destinations x + c_i: whole-row wall bounces carry the lid term with the push sign
    float sub[9];
    bool dwall[9];
    int drow[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        bool wall, top;
        drow[i] = src_row<EDGE>(l.y, -L::cy(i), ny, P.per[1], wall, top);
        dwall[i] = wall;
        sub[i] = (wall && top && L::cx(i) != 0) ? lid_term<L>(i, P.ulid) : 0.0f;
    }
    if (l.active) collide_lane<STORE, COLL, FORCE, EDGE, false>(P, v, lid, sub);
    const int own = l.y * nx + l.x0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const int cx = L::cx(i);
        E* plane = A + i * N + drow[i] * nx;
        E* bb = A + L::opp(i) * N + l.y * nx;  // own row, opposite slot
        if (dwall[i]) {
            if (l.active) st_plain(A + L::opp(i) * N + own, v[i]);
            continue;
        }
        if (cx == 0) {
            if (l.active) st_plain(plane + l.x0, v[i]);
        } else if (cx == 1) {
            const uint32_t up = from_prev<SEG>(l, elem<V>(v[i], V - 1));
            if (!l.active) continue;
            const uint4 su = shift_up<V>(v[i], up);
            if (!l.first || l.rot) st_plain(plane + l.x0, su);
            else st_tail<V>(plane + l.x0, su);  // slot x0 belongs to the previous warp
            if (l.last && !l.rot) {
                E* dst = l.x0 + V < nx ? plane + l.x0 + V
                                       : (P.per[0] ? plane : bb + nx - 1);
                st1(dst, elem<V>(v[i], V - 1));
            }
        } else {
            const uint32_t dn = from_next<SEG>(l, elem<V>(v[i], 0));
            if (!l.active) continue;
            const uint4 sd = shift_down<V>(v[i], dn);
            if (!l.last || l.rot) st_plain(plane + l.x0, sd);
            else st_head<V>(plane + l.x0, sd);  // slot x0 + V - 1 belongs to the next warp
            if (l.first && !l.rot) {
                E* dst = l.x0 > 0 ? plane + l.x0 - 1 : (P.per[0] ? plane + nx - 1 : bb);
                st1(dst, elem<V>(v[i], 0));
            }
        }
    }
}

template <int STORE, int COLL, bool FORCE, bool SEG>
__global__ void __launch_bounds__(kThreads)
k_d2q9_aa_odd(const StepParams P, void* Av) {
    using E = typename VT<STORE>::E;
    E* A = static_cast<E*>(Av);
    const Lane l = lane_of<STORE, SEG>(P);
    if (edge_warp<SEG>(P, l)) aa_odd_row<STORE, COLL, FORCE, true, SEG>(P, A, l);
    else aa_odd_row<STORE, COLL, FORCE, false, SEG>(P, A, l);
}

template <int STORE, int COLL, bool FORCE>
int go(const StepParams& P, const void* src, void* dst, int pattern, cudaStream_t s,
       bool staged) {
    constexpr int V = VT<STORE>::V;
    if (staged && pattern == LBM_PATTERN_AB)
        return go_staged<L, STORE, COLL, FORCE, LBM_PATTERN_AB>(P, src, dst, s);
    if (staged && pattern == LBM_PATTERN_AA_ODD)
        return go_staged<L, STORE, COLL, FORCE, LBM_PATTERN_AA_ODD>(P, dst, dst, s);
    if (pattern == LBM_PATTERN_AA_EVEN) {
        const int threads = P.N / V;
        k_d2q9_aa_even<STORE, COLL, FORCE>
            <<<(threads + kThreads - 1) / kThreads, kThreads, 0, s>>>(P, dst);
        return int(cudaGetLastError());
    }
    const int per_row = P.n[0] / V;
    if (per_row < kThreads) {  // rows of fewer than 128 lanes: several rows per block
        const dim3 block = block_for_rows(P.n[0], V);
        const dim3 grid((per_row + block.x - 1) / block.x, (P.n[1] + block.y - 1) / block.y);
        if (pattern == LBM_PATTERN_AB)
            k_d2q9_ab<STORE, COLL, FORCE, true><<<grid, block, 0, s>>>(P, src, dst);
        else
            k_d2q9_aa_odd<STORE, COLL, FORCE, true><<<grid, block, 0, s>>>(P, dst);
        return int(cudaGetLastError());
    }
    const dim3 grid((per_row + kThreads - 1) / kThreads, P.n[1]);
    if (pattern == LBM_PATTERN_AB)
        k_d2q9_ab<STORE, COLL, FORCE, false><<<grid, kThreads, 0, s>>>(P, src, dst);
    else
        k_d2q9_aa_odd<STORE, COLL, FORCE, false><<<grid, kThreads, 0, s>>>(P, dst);
    return int(cudaGetLastError());
}

template <int STORE, int COLL>
int go_f(const LbmDesc& d, const StepParams& P, const void* src, void* dst, int pattern,
         cudaStream_t s) {
    const bool staged = (d.flags & LBM_FLAG_STAGED) != 0;
    return needs_force(d) ? go<STORE, COLL, true>(P, src, dst, pattern, s, staged)
                          : go<STORE, COLL, false>(P, src, dst, pattern, s, staged);
}

template <int STORE>
int go_c(const LbmDesc& d, const StepParams& P, const void* src, void* dst, int pattern,
         cudaStream_t s) {
    switch (d.collision) {
        case LBM_BGK: return go_f<STORE, LBM_BGK>(d, P, src, dst, pattern, s);
        case LBM_TRT: return go_f<STORE, LBM_TRT>(d, P, src, dst, pattern, s);
        case LBM_MRT: return go_f<STORE, LBM_MRT>(d, P, src, dst, pattern, s);
        case LBM_STREAM_ONLY:
            return go<STORE, LBM_STREAM_ONLY, false>(P, src, dst, pattern, s,
                                                     (d.flags & LBM_FLAG_STAGED) != 0);
    }
    return LBM_E_COLLISION;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ------------------------------------------------------------------------- batched lattices
// One launch advances every lattice of a batch by one step. Each lattice's rows are laid end
// to end as one sequence of V-node vectors (nx / V per row); a work item is 32 consecutive
// vectors, one per lane, so rows narrower than a warp do not leave lanes idle. Lattice l owns
// items [item0_l, item0_l + ceil(nx ny / V / 32)). A warp reads its lattice's parameters from
// a per-item copy (one uniform load, no lattice lookup before it) and runs the single-lattice
// row code on that lattice's slice of the buffers: the lane at a row start, or at the warp start, takes its
// x-halo from memory instead of from its neighbour lane. A warp touching a row next to a y
// wall takes the general (wall and lid) path as a whole. PERSIST: a grid of a tuned size whose
// warps stride over the items; otherwise one item per warp (no loop state to keep, which
// leaves more registers to the collision).
//
// 16-bit batches collide the two nodes of a word together (packed f32x2, F2). 16-bit MRT
// batches are capped at 3 blocks of 256 threads per SM (80 registers): on the 64-cavity
// workload the packed MRT collision under that cap measured 155K MLUPS (0.86 of copy
// bandwidth) against 143-146K for the one-node form; 2 blocks per SM measured 139K, no cap
// 106K.
template <int STORE, int COLL, bool PERSIST>
__global__ void __launch_bounds__(256, (VT<STORE>::V == 8 && COLL == LBM_MRT) ? 3 : 1)
k_d2q9_batch_ab(const BatchLattice* __restrict__ item_tab, int items,
                const void* __restrict__ Av, void* __restrict__ Bv) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    const E* __restrict__ A = static_cast<const E*>(Av);
    E* __restrict__ B = static_cast<E*>(Bv);
    const int lane = threadIdx.x & 31;
    const int stride = PERSIST ? (gridDim.x * blockDim.x) >> 5 : items;
    for (int item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < items;
         item += stride) {
        const BatchLattice& bl = item_tab[item];
        const int local = item - __ldg(&bl.item0);
        const int vrow = __ldg(&bl.segs);  // vectors per row
        StepParams P;
        P.n[0] = __ldg(&bl.nx);
        P.n[1] = __ldg(&bl.ny);
        P.n[2] = 1;
        P.N = P.n[0] * P.n[1];
        const int per = __ldg(&bl.periodic_mask);
        P.per[0] = per & 1;
        P.per[1] = (per >> 1) & 1;
        P.per[2] = 1;
        P.ulid = __ldg(&bl.ulid);
        P.F[0] = P.F[1] = P.F[2] = 0.0f;
        P.r0 = __ldg(&bl.r0);
        P.r1 = __ldg(&bl.r1);
        P.r2 = __ldg(&bl.r2);
        P.r3 = __ldg(&bl.r3);
        P.solid = nullptr;
        P.field = nullptr;
        P.mx = nullptr;
        P.inlet = nullptr;
        P.outlet = 0;
        const int vidx = local * 32 + lane;
        const int nvec = vrow * P.n[1];
        Lane l;
        l.sl = lane;
        l.w = 32;
        l.rot = false;
        l.active = vidx < nvec;
        // row of the lane's vector: from the item's first row, a few whole rows further
        int xv = __ldg(&bl.xv0) + lane, y = __ldg(&bl.y0);
        while (xv >= vrow) {
            xv -= vrow;
            ++y;
        }
        l.y = l.active ? y : 0;
        l.x0 = l.active ? xv * V : 0;
        l.first = lane == 0 || l.x0 == 0;
        l.last = l.active && (lane == 31 || l.x0 + V >= P.n[0] || vidx + 1 >= nvec);
        const long long base = __ldg(&bl.base);
        const bool edge = __any_sync(0xffffffffu, l.active && edge_row(P, l.y));
        constexpr bool pack = VT<STORE>::V == 8;
        if (edge) ab_row<STORE, COLL, false, true, pack>(P, A + base, B + base, l);
        else ab_row<STORE, COLL, false, false, pack>(P, A + base, B + base, l);
    }
}

template <int STORE, bool PERSIST>
int batch_go(int collision, const BatchLattice* item_tab, int items, const void* src,
             void* dst, int grid, int block, cudaStream_t s) {
    switch (collision) {
        case LBM_BGK:
            k_d2q9_batch_ab<STORE, LBM_BGK, PERSIST>
                <<<grid, block, 0, s>>>(item_tab, items, src, dst);
            break;
        case LBM_TRT:
            k_d2q9_batch_ab<STORE, LBM_TRT, PERSIST>
                <<<grid, block, 0, s>>>(item_tab, items, src, dst);
            break;
        case LBM_MRT:
            k_d2q9_batch_ab<STORE, LBM_MRT, PERSIST>
                <<<grid, block, 0, s>>>(item_tab, items, src, dst);
            break;
        default:
            return LBM_E_COLLISION;
    }
    return int(cudaGetLastError());
}

template <int STORE>
int batch_go_p(int collision, const BatchLattice* item_tab, int items, const void* src,
               void* dst, int grid, int block, bool persist, cudaStream_t s) {
    return persist ? batch_go<STORE, true>(collision, item_tab, items, src, dst, grid, block, s)
                   : batch_go<STORE, false>(collision, item_tab, items, src, dst, grid, block, s);
}

}  // namespace

int launch_batch_d2q9(int collision, int storage, const BatchLattice* item_tab, int items,
                      const void* src, void* dst, int grid, int block, bool persist,
                      cudaStream_t s) {
    switch (storage) {
        case LBM_STORE_F32:
            return batch_go_p<LBM_STORE_F32>(collision, item_tab, items, src, dst, grid,
                                             block, persist, s);
        case LBM_STORE_F32_SHIFTED:
            return batch_go_p<LBM_STORE_F32_SHIFTED>(collision, item_tab, items, src, dst, grid,
                                                     block, persist, s);
        case LBM_STORE_F16:
            return batch_go_p<LBM_STORE_F16>(collision, item_tab, items, src, dst, grid,
                                             block, persist, s);
        case LBM_STORE_BF16:
            return batch_go_p<LBM_STORE_BF16>(collision, item_tab, items, src, dst, grid,
                                              block, persist, s);
    }
    return LBM_E_STORAGE;
}

int launch_fast_d2q9(const LbmDesc& d, const void* src, void* dst, int pattern,
                     cudaStream_t s) {
    // the vector kernels cover box problems whose rows split into whole 16-byte vectors
    if (d.solid_bits || d.force_field || d.mx_force || d.inlet_u || d.outlet) return 1;
    const int V = (d.storage == LBM_STORE_F16 || d.storage == LBM_STORE_BF16) ? 8 : 4;
    if (d.nx % V != 0) return 1;
    if (!aligned16(src) || !aligned16(dst)) return 1;
    const StepParams P = make_params(d);
    switch (d.storage) {
        case LBM_STORE_F32: return go_c<LBM_STORE_F32>(d, P, src, dst, pattern, s);
        case LBM_STORE_F32_SHIFTED: return go_c<LBM_STORE_F32_SHIFTED>(d, P, src, dst, pattern, s);
        case LBM_STORE_F16: return go_c<LBM_STORE_F16>(d, P, src, dst, pattern, s);
        case LBM_STORE_BF16: return go_c<LBM_STORE_BF16>(d, P, src, dst, pattern, s);
    }
    return LBM_E_STORAGE;
}

}  // namespace lbm
