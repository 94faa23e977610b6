// TMA-staged fused step: persistent CTAs, one producer warp, a ring of shared-memory stages.
//
// A work item is one row segment (x0 .. x0 + wlen - 1 at fixed y, z). For every population
// plane one lane of the producer warp copies the pulled source row segment -- row
// (y - c_iy, z - c_iz), wrapped or, behind a wall, the node row of the opposite plane -- into
// the stage with one contiguous cp.async.bulk copy that, inside the row, already includes the
// 16-byte halo chunk its x-shift needs; the single element beyond a row end (periodic wrap or
// x wall) is read from global memory by the consumer lane of that node. Completion is
// counted in bytes on the stage's `full` mbarrier; consumer warps read each node's 19 (or 9)
// values at the shifted position x - c_ix from shared memory (consecutive lanes, consecutive
// words: no bank conflicts), collide, and store coalesced rows straight to global memory, then
// release the stage on its `empty` mbarrier. The loads thus run up to stages-1 rows ahead of
// the arithmetic without holding registers, so the memory-level parallelism does not depend
// on how the compiler schedules the consumers.
//
// Patterns: AB (pull src -> dst) and AA-odd (pull from the swapped slots, push each node's
// results to x + c_i one node at a time, which keeps every slot owned by one node). Walls, the
// lid term and the x wrap follow step_generic.cuh. Every mbarrier wait is bounded: on timeout
// the thread sets bit 1 of the device error word and returns (the producer issues nothing
// more, so no copy is left in flight into a stage no one waits for).
#pragma once

#include "codec.cuh"
#include "collide.cuh"
#include "lattice.cuh"
#include "params.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace lbm {

struct StagedCfg {
    int W;              // segment width in nodes (multiple of 16 bytes worth of elements)
    int segs;           // segments per row
    int items;          // segs * ny * nz
    int stages;         // ring depth
    int cons_warps;     // consumer warps per CTA
    int no_issue;       // test mode: the producer issues no copy, so every consumer wait runs out
    unsigned long long timeout_ns;
    unsigned int* err;  // device error word
};

constexpr unsigned int kDevErrTimeout = 1u;

__host__ __device__ constexpr int staged_barrier_bytes(int stages) {
    return ((2 * stages * 8 + 127) / 128) * 128;
}

// Pull source of direction i for node row (y, z): wall = behind a y or z wall; top = behind
// the top wall of the last axis. The x axis is resolved per node.
template <class L>
__device__ __forceinline__ void staged_src_row(const StepParams& P, int i, int y, int z, int& ys,
                                               int& zs, bool& wall, bool& top) {
    wall = top = false;
    ys = y - L::cy(i);
    zs = z - L::cz(i);
    if (ys < 0 || ys >= P.n[1]) {
        if (P.per[1]) ys += ys < 0 ? P.n[1] : -P.n[1];
        else { wall = true; if (L::D == 2 && ys >= P.n[1]) top = true; }
    }
    if (L::D == 3 && (zs < 0 || zs >= P.n[2])) {
        if (P.per[2]) zs += zs < 0 ? P.n[2] : -P.n[2];
        else { wall = true; if (zs >= P.n[2]) top = true; }
    }
}

// Lane `lane` of the producer warp issues the one copy of plane `lane` (lanes >= Q idle):
// the source row segment including, inside the row, the 16-byte halo chunk its x-shift needs.
// The element beyond a row end (periodic wrap or x wall) is not copied; the consumer lane of
// that node reads it from global memory. Returns the bytes this lane announced.
template <class L, int STORE, int PATTERN>
__device__ __forceinline__ void staged_issue(const StepParams& P, const StagedCfg& C,
                                             const typename VT<STORE>::E* A,
                                             typename VT<STORE>::E* st, uint64_t* bar, int item,
                                             int lane) {
    using E = typename VT<STORE>::E;
    constexpr int H = 16 / int(sizeof(E));
    if (lane >= L::Q) return;
    const int i = lane;
    const int nx = P.n[0], ny = P.n[1], N = P.N;
    const int seg = item % C.segs, row = item / C.segs;
    const int y = row % ny, z = row / ny;
    const int x0 = seg * C.W;
    const int wlen = min(C.W, nx - x0);
    const int pitch = C.W + 2 * H;
    const int src_slot = PATTERN == LBM_PATTERN_AB ? i : L::opp(i);
    const int bb_slot = PATTERN == LBM_PATTERN_AB ? L::opp(i) : i;
    int ys, zs;
    bool wall, top;
    staged_src_row<L>(P, i, y, z, ys, zs, wall, top);
    E* dst = st + i * pitch + H;
    const E* src;
    int n = wlen;
    if (wall) {
        src = A + bb_slot * N + (y + ny * z) * nx + x0;
    } else {
        src = A + src_slot * N + (ys + ny * zs) * nx + x0;
        const int cx = L::cx(i);
        if (cx == 1 && x0 > 0) {  // node x pulls x - 1: left halo chunk
            src -= H;
            dst -= H;
            n += H;
        } else if (cx == -1 && x0 + wlen < nx) {  // node x pulls x + 1: right halo chunk
            n += H;
        }
    }
    const uint32_t bytes = uint32_t(n) * uint32_t(sizeof(E));
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    bulk_load(dst, src, bytes, bar);
}

template <class L, int STORE, int COLL, bool FORCE, int PATTERN>
__global__ void __launch_bounds__(32 * 9)
k_staged(const StepParams P, const StagedCfg C, const typename VT<STORE>::E* A,
         typename VT<STORE>::E* B) {
    using E = typename VT<STORE>::E;
    using T = VT<STORE>;
    constexpr int H = 16 / int(sizeof(E));
    constexpr int Q = L::Q;
    constexpr bool SHIFT = Codec<STORE>::shifted;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + C.stages;
    E* ring = reinterpret_cast<E*>(smem + staged_barrier_bytes(C.stages));
    const int pitch = C.W + 2 * H;
    const int stage_elems = Q * pitch;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ncw = C.cons_warps;
    if (threadIdx.x == 0) {
        for (int s = 0; s < C.stages; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, ncw);
        }
        mbar_init_fence();
    }
    __syncthreads();

    if (warp == ncw) {  // ------------------------------------------------ producer
        if (C.no_issue) return;
        int it = 0;
        for (int item = blockIdx.x; item < C.items; item += gridDim.x, ++it) {
            const int s = it % C.stages;
            const uint32_t ph = (it / C.stages) & 1;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(empty + s, ph ^ 1u, C.timeout_ns);
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) {
                    atomicOr(C.err, kDevErrTimeout);
                    // let the copies this warp issued for the other slots land before the
                    // block can exit (each wait bounded again; the error is already set)
                    for (int k = it - C.stages + 1; k < it; ++k)
                        if (k >= 0)
                            mbar_wait(full + k % C.stages, (k / C.stages) & 1, C.timeout_ns);
                }
                return;
            }
            fence_proxy_async();
            staged_issue<L, STORE, PATTERN>(P, C, A, ring + s * stage_elems, full + s, item, lane);
            __syncwarp();  // every lane's expect_tx precedes the phase-completing arrival
            if (lane == 0) mbar_arrive(full + s);
        }
        return;
    }

    // ------------------------------------------------------------------- consumers
    const int nx = P.n[0], ny = P.n[1], N = P.N;
    const int nct = ncw * 32;
    int it = 0;
    for (int item = blockIdx.x; item < C.items; item += gridDim.x, ++it) {
        const int s = it % C.stages;
        const uint32_t ph = (it / C.stages) & 1;
        if (!mbar_wait(full + s, ph, C.timeout_ns)) {
            atomicOr(C.err, kDevErrTimeout);
            return;
        }
        const int seg = item % C.segs, row = item / C.segs;
        const int y = row % ny, z = row / ny;
        const int x0 = seg * C.W;
        const int wlen = min(C.W, nx - x0);
        const E* st = ring + s * stage_elems;
        for (int xl = threadIdx.x; xl < wlen; xl += nct) {
            const int x = x0 + xl;
            const int n = x + nx * (y + ny * z);
            float f[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) {
                const int cx = L::cx(i);
                int ys, zs;
                bool wall, top;
                staged_src_row<L>(P, i, y, z, ys, zs, wall, top);
                uint32_t raw;
                if (!wall && ((cx == 1 && x == 0) || (cx == -1 && x == nx - 1))) {
                    // the source lies beyond a row end: wrapped (periodic x) or, behind an x
                    // wall, the node's own opposite slot
                    const int src_slot = PATTERN == LBM_PATTERN_AB ? i : L::opp(i);
                    const int bb_slot = PATTERN == LBM_PATTERN_AB ? L::opp(i) : i;
                    raw = P.per[0] ? uint32_t(A[src_slot * N + (ys + ny * zs) * nx +
                                                (cx == 1 ? nx - 1 : 0)])
                                   : uint32_t(A[bb_slot * N + n]);
                } else {
                    raw = uint32_t(st[i * pitch + H + xl - (wall ? 0 : cx)]);
                }
                f[i] = T::f(raw);
                if (wall && top && cx != 0) f[i] = add_lid(f[i], lid_term<L>(i, P.ulid));
            }
            const float F[3] = {P.F[0], P.F[1], P.F[2]};
            collide<L, COLL, SHIFT, FORCE, Codec<STORE>::compact>(f, F, P.r0, P.r1, P.r2, P.r3);
            if (PATTERN == LBM_PATTERN_AB) {
#pragma unroll
                for (int i = 0; i < Q; ++i) __stcs(B + i * N + n, static_cast<E>(T::b(f[i])));
            } else {  // AA odd: push to x + c_i, or bounce into the own slot opp(i)
                const int crd[3] = {x, y, z};
#pragma unroll
                for (int i = 0; i < Q; ++i) {
                    bool wall = false, top = false;
                    int off = 0, stride = 1;
#pragma unroll
                    for (int a = 0; a < L::D; ++a) {
                        const int c = cc<L>(i, a);
                        if (c != 0) {
                            int d = crd[a] + c;
                            if (d < 0 || d >= P.n[a]) {
                                if (P.per[a]) d += d < 0 ? P.n[a] : -P.n[a];
                                else { wall = true; if (a == L::D - 1 && d >= P.n[a]) top = true; }
                            }
                            off += (d - crd[a]) * stride;
                        }
                        stride *= P.n[a];
                    }
                    if (wall) {
                        float v = f[i];
                        if (top && L::cx(i) != 0) v = sub_lid(v, lid_term<L>(i, P.ulid));
                        B[L::opp(i) * N + n] = static_cast<E>(T::b(v));
                    } else {
                        B[i * N + n + off] = static_cast<E>(T::b(f[i]));
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
    }
}

}  // namespace lbm
