// Vectorised D3Q19 register kernels: the D2Q9 row design (step_d2q9.cu) over rows (y, z).
//
// Every lane owns V consecutive nodes of one row (16 bytes per plane: 4 fp32 or 8 x 16-bit);
// the 19 source row segments are read with aligned 16-byte loads at rows (y - c_iy, z - c_iz),
// shifted along x in registers with one warp shuffle per x-moving plane, and the two halo
// elements of a row segment are scalar loads (none when the segment is a whole periodic row).
// A row of 32 lanes or more spans whole warps (block (lanes_x, rows), lanes_x a multiple of
// 32); a shorter row takes a power-of-two segment of w lanes and a warp holds 32 / w rows,
// its shuffles running within segments of width w. Rows next to a y or z wall take a general
// path with the wall and lid logic; all other rows run without it (the choice is made per
// warp, so that no shuffle runs in divergent code).
#pragma once

#include "codec.cuh"
#include "collide.cuh"
#include "lattice.cuh"
#include "params.cuh"
#include "vec.cuh"

namespace lbm {
namespace rows3d {

using L = D3Q19;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kThreads = 128;

// Source row (y - cy, z - cz), wrapped; EDGE rows report walls (then not wrapped) and top.
template <bool EDGE>
__device__ __forceinline__ int src_row(const StepParams& P, int y, int z, int cy, int cz,
                                       bool& wall, bool& top) {
    int ys = y - cy, zs = z - cz;
    wall = top = false;
    if constexpr (!EDGE) {
        ys += ys < 0 ? P.n[1] : (ys >= P.n[1] ? -P.n[1] : 0);
        zs += zs < 0 ? P.n[2] : (zs >= P.n[2] ? -P.n[2] : 0);
    } else {
        if (ys < 0 || ys >= P.n[1]) {
            if (P.per[1]) ys += ys < 0 ? P.n[1] : -P.n[1];
            else wall = true;
        }
        if (zs < 0 || zs >= P.n[2]) {
            if (P.per[2]) zs += zs < 0 ? P.n[2] : -P.n[2];
            else { wall = true; top = zs >= P.n[2]; }
        }
    }
    return ys + P.n[1] * zs;
}

// w: lanes of a row segment (32, or the power of two a shorter row is given); sl: the lane's
// index in it. rot: the segment holds one whole periodic row (nx = w V), so the x neighbours
// across the row's ends are its last and first lanes: shifts rotate within the segment, with
// no halo loads and no partial stores at the row's ends. D3Q19 256^3 (fp16 / bf16) and 128^3
// (fp32) measured 0.898 -> 0.923 (AB fp16), 0.825 -> 0.844 (AA fp16), 0.851 -> 0.912 (AA fp32
// 128^3).
struct Lane3 {
    int x0, y, z, sl, w;
    bool active, first, last, rot;
};

// SEG: the block may hold rows of fewer than 32 lanes (w from the block shape); otherwise w is
// the constant 32 and the shuffles compile to their whole-warp form (the runtime width cost
// ~1.3 % at 256^3 fp16, where every row spans whole warps).
template <int V, bool SEG>
__device__ __forceinline__ Lane3 lane_of(const StepParams& P) {
    Lane3 l;
    l.w = (SEG && blockDim.x < 32) ? int(blockDim.x) : 32;
    l.sl = threadIdx.x & (l.w - 1);
    l.x0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    l.y = blockIdx.y * blockDim.y + threadIdx.y;
    l.z = blockIdx.z;
    l.active = l.x0 < P.n[0] && l.y < P.n[1];
    l.first = l.sl == 0;
    l.last = l.active && (l.sl == l.w - 1 || l.x0 + V >= P.n[0]);
    l.rot = P.per[0] && P.n[0] == l.w * V;
    return l;
}

// The value of lane sl - 1 (up) or sl + 1 (dn) of the segment, cyclically.
__device__ __forceinline__ uint32_t from_prev(const Lane3& l, uint32_t x) {
    return __shfl_sync(kFull, x, (l.sl + l.w - 1) & (l.w - 1), l.w);
}
__device__ __forceinline__ uint32_t from_next(const Lane3& l, uint32_t x) {
    return __shfl_sync(kFull, x, (l.sl + 1) & (l.w - 1), l.w);
}

__device__ __forceinline__ bool edge_row(const StepParams& P, int y, int z) {
    return (!P.per[1] && (y == 0 || y == P.n[1] - 1)) ||
           (!P.per[2] && (z == 0 || z == P.n[2] - 1));
}

// Whether the warp takes the wall path: any of its rows is next to a y or z wall (all 32 lanes
// call this, before any of them can leave).
template <bool SEG>
__device__ __forceinline__ bool edge_warp(const StepParams& P, const Lane3& l) {
    const bool e = edge_row(P, l.y, l.z);
    if constexpr (SEG) return l.w < 32 ? __any_sync(kFull, e) : e;
    else return e;
}

template <int STORE, bool READ_OPP, bool NC, bool EDGE>
__device__ __forceinline__ void pull_rows(const StepParams& P, const typename VT<STORE>::E* A,
                                          const Lane3& l, uint4 (&v)[19], float (&lid)[19]) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    const int nx = P.n[0], N = P.N;
    const int own_row = l.y + P.n[1] * l.z;
    uint32_t halo[19];
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const int cx = L::cx(i);
        const int src_slot = READ_OPP ? L::opp(i) : i;
        const int bb_slot = READ_OPP ? i : L::opp(i);
        bool wall, top;
        const int r = src_row<EDGE>(P, l.y, l.z, L::cy(i), L::cz(i), wall, top);
        lid[i] = (wall && top && cx != 0) ? lid_term<L>(i, P.ulid) : 0.0f;
        v[i] = make_uint4(0u, 0u, 0u, 0u);
        halo[i] = 0u;
        if (!l.active) continue;
        if (wall) {
            const E* p = A + bb_slot * N + own_row * nx + l.x0;
            v[i] = NC ? ld_nc(p) : ld_plain(p);
            continue;
        }
        const E* row = A + src_slot * N + r * nx;
        v[i] = NC ? ld_nc(row + l.x0) : ld_plain(row + l.x0);
        if (cx == 1 && l.first && !l.rot) {
            const E* h = l.x0 > 0 ? row + l.x0 - 1
                                  : (P.per[0] ? row + nx - 1 : A + bb_slot * N + own_row * nx);
            halo[i] = NC ? ld1_nc(h) : ld1(h);
        }
        if (cx == -1 && l.last && !l.rot) {
            const E* h = l.x0 + V < nx ? row + l.x0 + V
                                       : (P.per[0] ? row : A + bb_slot * N + own_row * nx + nx - 1);
            halo[i] = NC ? ld1_nc(h) : ld1(h);
        }
    }
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const int cx = L::cx(i);
        if (cx == 0) continue;
        bool wall, top;
        src_row<EDGE>(P, l.y, l.z, L::cy(i), L::cz(i), wall, top);
        if (cx == 1) {
            uint32_t up = from_prev(l, elem<V>(v[i], V - 1));
            if (l.first && !l.rot) up = halo[i];
            if (!wall) v[i] = shift_up<V>(v[i], up);
        } else {
            uint32_t dn = from_next(l, elem<V>(v[i], 0));
            if (l.last && !l.rot) dn = halo[i];
            if (!wall) v[i] = shift_down<V>(v[i], dn);
        }
    }
}

// Collide the V nodes of the lane in place. With LIDS, lid[i] is added to the pulled value of
// direction i and sub[i] is subtracted from its post-collision value (the AA-odd push into
// the lid). 16-bit storages: PACK collides the two nodes of a word together with packed f32x2
// instructions (F2), else one after the other (F1); the results are identical. Under the same
// 128-register cap (4 blocks per SM) packing measured faster for the pull kernel (D3Q19 256^3
// TRT AB: fp16 0.923 -> 0.939 of copy, bf16 0.900 -> 0.937) and slower for the AA-odd push
// kernel, which also holds its push state (fp16 0.844 -> 0.817).
template <int STORE, int COLL, bool FORCE, bool LIDS, bool PACK>
__device__ __forceinline__ void collide_lane(const StepParams& P, uint4 (&v)[19],
                                             const float (&lid)[19], const float (&sub)[19]) {
    using T = VT<STORE>;
    constexpr int V = T::V;
    const float F[3] = {P.F[0], P.F[1], P.F[2]};
    if constexpr (COLL == LBM_MRT) {
        // One copy of the moment transform per kernel (8 unrolled copies made one translation
        // unit take half an hour to compile): a rolled loop over the lane's nodes collides
        // element 0 and rotates every vector down by one element, appending the result, so
        // after V passes each result sits in its node's place.
#pragma unroll 1
        for (int k = 0; k < V; ++k) {
            float f[19];
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                f[i] = T::f(elem<V>(v[i], 0));
                if (LIDS) f[i] = add_lid(f[i], lid[i]);
            }
            collide<L, LBM_MRT, Codec<STORE>::shifted, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 19; ++i)
                v[i] = shift_down<V>(v[i], T::b(LIDS ? sub_lid(f[i], sub[i]) : f[i]));
        }
    } else if constexpr (V == 4) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            float f[19];
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                f[i] = T::f(elem<V>(v[i], k));
                if (LIDS) f[i] = add_lid(f[i], lid[i]);
            }
            collide<L, COLL, Codec<STORE>::shifted, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 19; ++i) put<V>(v[i], k, T::b(LIDS ? sub_lid(f[i], sub[i]) : f[i]));
        }
    } else if constexpr (PACK) {  // 16-bit: the two nodes of a word at once
#pragma unroll
        for (int jw = 0; jw < 4; ++jw) {
            F2 f[19];
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                f[i].v = unpack2<STORE>(word(v[i], jw));
                if (LIDS) f[i] = add_lid(f[i], lid[i]);
            }
            collide2<L, COLL, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                if (LIDS) f[i] = sub_lid(f[i], sub[i]);
                set_word(v[i], jw, pack2<STORE>(f[i].v.x, f[i].v.y));
            }
        }
    } else {
        // 16-bit: two nodes per word, packed conversions, the two nodes collided one after the
        // other (F1 arithmetic, bit-for-bit the packed F2 result).
#pragma unroll
        for (int jw = 0; jw < 4; ++jw) {
            float f0[19], f1[19];
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                const float2 p = unpack2<STORE>(word(v[i], jw));
                f0[i] = LIDS ? add_lid(p.x, lid[i]) : p.x;
                f1[i] = LIDS ? add_lid(p.y, lid[i]) : p.y;
            }
            collide<L, COLL, Codec<STORE>::shifted, FORCE, true>(f0, F, P.r0, P.r1, P.r2, P.r3);
            collide<L, COLL, Codec<STORE>::shifted, FORCE, true>(f1, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < 19; ++i)
                set_word(v[i], jw, LIDS ? pack2<STORE>(sub_lid(f0[i], sub[i]),
                                                       sub_lid(f1[i], sub[i]))
                                        : pack2<STORE>(f0[i], f1[i]));
        }
    }
}

template <int STORE, int COLL, bool FORCE, bool EDGE>
__device__ __forceinline__ void ab_row(const StepParams& P, const typename VT<STORE>::E* A,
                                       typename VT<STORE>::E* B, const Lane3& l) {
    uint4 v[19];
    float lid[19];
    pull_rows<STORE, false, true, EDGE>(P, A, l, v, lid);
    if (!l.active) return;
    const float zero[19] = {};
    collide_lane<STORE, COLL, FORCE, EDGE, !FORCE>(P, v, lid, zero);
    const int n0 = (l.y + P.n[1] * l.z) * P.n[0] + l.x0;
#pragma unroll
    for (int i = 0; i < 19; ++i) st_cs(B + i * P.N + n0, v[i]);
}

// 16-bit without a body force: capped at 128 registers (4 blocks per SM), with packed
// collisions; left free the kernel takes ~158 registers and 3 blocks, and this latency-bound
// kernel measured 79.5K instead of 72.5K MLUPS (256^3 TRT fp16, one-node collisions). The
// forced variants would spill several hundred bytes under the cap and keep one-node
// collisions.
template <int STORE, int COLL, bool FORCE, bool SEG>
__global__ void __launch_bounds__(kThreads,
                                  (VT<STORE>::V == 8 && !FORCE && COLL != LBM_MRT) ? 4 : 1)
k_ab(const StepParams P, const void* __restrict__ Av, void* __restrict__ Bv) {
    using E = typename VT<STORE>::E;
    const E* __restrict__ A = static_cast<const E*>(Av);
    E* __restrict__ B = static_cast<E*>(Bv);
    const Lane3 l = lane_of<VT<STORE>::V, SEG>(P);
    if (edge_warp<SEG>(P, l)) ab_row<STORE, COLL, FORCE, true>(P, A, B, l);
    else ab_row<STORE, COLL, FORCE, false>(P, A, B, l);
}

// AA odd step in place (the D2Q9 design of step_d2q9.cu over rows (y, z)): pull from the
// swapped slots A[opp(i), x - c_i] (bounce-back: A[i, x]), collide, push p_i to
// A[i, x + c_i] or, behind a wall, to the node's own slot A[opp(i), x] minus the lid term.
// Every slot is read and written by one node only (slot (i, x + c_i) belongs to node x), so
// a lane stores an aligned vector only where all its elements belong to nodes of its own
// warp, which loaded before any lane of the warp stores; a warp-edge lane stores the V - 1
// slots of its own nodes in three aligned pieces (st_tail / st_head).
template <int STORE, int COLL, bool FORCE, bool EDGE>
__device__ __forceinline__ void aa_odd_row(const StepParams& P, typename VT<STORE>::E* A,
                                           const Lane3& l) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    const int nx = P.n[0], N = P.N;
    uint4 v[19];
    float lid[19], sub[19];
    pull_rows<STORE, true, false, EDGE>(P, A, l, v, lid);
#pragma unroll
    for (int i = 0; i < 19; ++i) {  // pushes bouncing off the lid carry its term, negated
        bool wall, top;
        src_row<EDGE>(P, l.y, l.z, -L::cy(i), -L::cz(i), wall, top);
        sub[i] = (wall && top && L::cx(i) != 0) ? lid_term<L>(i, P.ulid) : 0.0f;
    }
    if (l.active) collide_lane<STORE, COLL, FORCE, EDGE, false>(P, v, lid, sub);
    // an opaque zero computed from the collision's output: the push addresses below depend on
    // it, so the compiler forms them after the collision instead of holding all 19 through it.
    // With it the kernel fits 4 blocks per SM (128 registers, 32-40 bytes of spills instead of
    // ~375): D3Q19 AA at 256^3 measured 0.909 -> 0.944 of copy bandwidth (fp32), 0.767 ->
    // 0.816 (fp16)
    uint32_t z;
    asm("and.b32 %0, %1, 0;" : "=r"(z) : "r"(v[0].x));
    const int own_row = l.y + P.n[1] * l.z + int(z);
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const int cx = L::cx(i);
        bool wall, top;
        const int r = src_row<EDGE>(P, l.y, l.z, -L::cy(i), -L::cz(i), wall, top);
        E* plane = A + i * N + r * nx;
        E* bb = A + L::opp(i) * N + own_row * nx;  // own row, opposite slot
        if (wall) {
            if (l.active) st_plain(bb + l.x0, v[i]);
            continue;
        }
        if (cx == 0) {
            if (l.active) st_plain(plane + l.x0, v[i]);
        } else if (cx == 1) {
            const uint32_t up = from_prev(l, elem<V>(v[i], V - 1));
            if (!l.active) continue;
            const uint4 su = shift_up<V>(v[i], up);
            if (!l.first || l.rot) st_plain(plane + l.x0, su);
            else st_tail<V>(plane + l.x0, su);  // slot x0 belongs to the previous warp
            if (l.last && !l.rot) {
                E* dst = l.x0 + V < nx ? plane + l.x0 + V : (P.per[0] ? plane : bb + nx - 1);
                st1(dst, elem<V>(v[i], V - 1));
            }
        } else {
            const uint32_t dn = from_next(l, elem<V>(v[i], 0));
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
__global__ void __launch_bounds__(kThreads, COLL == LBM_MRT ? 1 : 4)
k_aa_odd(const StepParams P, void* Av) {
    using E = typename VT<STORE>::E;
    E* A = static_cast<E*>(Av);
    const Lane3 l = lane_of<VT<STORE>::V, SEG>(P);
    if (edge_warp<SEG>(P, l)) aa_odd_row<STORE, COLL, FORCE, true>(P, A, l);
    else aa_odd_row<STORE, COLL, FORCE, false>(P, A, l);
}

// Block shape (lanes along x, rows) for rows of nx nodes; SEG: rows of fewer than 32 lanes take
// power-of-two segments of a warp (else a whole warp, the rest of it idle).
inline dim3 block_for_rows(int nx, int V, bool seg) {
    const int need = (nx + V - 1) / V;
    if (seg && need < 32) {  // a power-of-two segment per row, 32 / w rows per warp
        int w = 1;
        while (w < need) w <<= 1;
        return dim3(w, kThreads / w);
    }
    int lanes = (need + 31) / 32 * 32;
    if (lanes > kThreads) lanes = kThreads;
    return dim3(lanes, kThreads / lanes);
}

// Whether a launch takes the segmented kernel: rows of fewer than 32 lanes, and every MRT or
// forced launch (those keep one instantiation each, to bound the compile time: MRT is
// compute-bound, and forced steps are not the throughput configurations).
template <int COLL, bool FORCE>
inline bool use_seg(int nx, int V) {
    return COLL == LBM_MRT || FORCE || (nx + V - 1) / V < 32;
}

template <int STORE, int COLL, bool FORCE>
int go_ab(const StepParams& P, const void* src, void* dst, cudaStream_t s) {
    constexpr int V = VT<STORE>::V;
    constexpr bool kOnlySeg = COLL == LBM_MRT || FORCE;
    const bool seg = use_seg<COLL, FORCE>(P.n[0], V);
    const dim3 block = block_for_rows(P.n[0], V, seg);
    const dim3 grid((P.n[0] / V + block.x - 1) / block.x, (P.n[1] + block.y - 1) / block.y,
                    P.n[2]);
    if (seg || kOnlySeg) k_ab<STORE, COLL, FORCE, true><<<grid, block, 0, s>>>(P, src, dst);
    else k_ab<STORE, COLL, FORCE, kOnlySeg><<<grid, block, 0, s>>>(P, src, dst);
    return int(cudaGetLastError());
}

template <int STORE, int COLL, bool FORCE>
int go_aa_odd(const StepParams& P, void* buf, cudaStream_t s) {
    constexpr int V = VT<STORE>::V;
    constexpr bool kOnlySeg = COLL == LBM_MRT || FORCE;
    const bool seg = use_seg<COLL, FORCE>(P.n[0], V);
    const dim3 block = block_for_rows(P.n[0], V, seg);
    const dim3 grid((P.n[0] / V + block.x - 1) / block.x, (P.n[1] + block.y - 1) / block.y,
                    P.n[2]);
    if (seg || kOnlySeg) k_aa_odd<STORE, COLL, FORCE, true><<<grid, block, 0, s>>>(P, buf);
    else k_aa_odd<STORE, COLL, FORCE, kOnlySeg><<<grid, block, 0, s>>>(P, buf);
    return int(cudaGetLastError());
}

}  // namespace rows3d
}  // namespace lbm
