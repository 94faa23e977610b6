// TMA-staged D3Q19 pull step for 16-bit storages on fully periodic lattices, whole rows per
// work item, two nodes per consumer thread.
//
// A work item is one whole row (y, z). The producer warp (one lane per plane, the copy code
// of step_staged.cuh) stages the 19 pulled source rows -- rows (y - c_iy, z - c_iz), wrapped --
// into a ring of shared-memory stages with one cp.async.bulk each, completing on the stage's
// `full` mbarrier. Consumer thread t owns nodes x = 2t, 2t + 1 (one 32-bit storage word per
// plane): it reads the word of each plane at x - c_ix straight from shared memory (one
// aligned 32-bit load for c_ix = 0; two and one byte permutation for c_ix = +-1, the periodic
// wrap being the row's other end, which is in the same stage), releases the stage on `empty`,
// collides its two nodes together with packed f32x2 arithmetic and stores one 32-bit word per
// plane. No row data is held in registers while the loads are in flight, and each node costs
// about half the instructions of the register row kernel's one-node collisions. Waits are
// bounded as in step_staged.cuh.
#pragma once

#include "codec.cuh"
#include "collide.cuh"
#include "dispatch.cuh"
#include "step_staged.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace lbm {

template <int STORE, int COLL, bool FORCE>
__global__ void __launch_bounds__(32 * 9)
k_staged_rows16(const StepParams P, const StagedCfg C, const uint16_t* A, uint16_t* B) {
    using L = D3Q19;
    constexpr int H = 8;  // halo elements of a stage row (16 bytes)
    constexpr int Q = 19;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + C.stages;
    uint16_t* ring = reinterpret_cast<uint16_t*>(smem + staged_barrier_bytes(C.stages));
    const int nx = P.n[0];
    const int pitch = nx + 2 * H;
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
                    for (int k = it - C.stages + 1; k < it; ++k)
                        if (k >= 0)
                            mbar_wait(full + k % C.stages, (k / C.stages) & 1, C.timeout_ns);
                }
                return;
            }
            fence_proxy_async();
            staged_issue<L, STORE, LBM_PATTERN_AB>(P, C, A, ring + s * stage_elems, full + s,
                                                   item, lane);
            __syncwarp();
            if (lane == 0) mbar_arrive(full + s);
        }
        return;
    }

    // ------------------------------------------------------------------- consumers
    const int t = threadIdx.x;       // pair index: nodes 2t, 2t + 1 of the row
    const int half = nx >> 1;        // words per stage row
    const int cur = (H >> 1) + t;    // word offsets inside a stage row
    const int prev = (H >> 1) + (t == 0 ? half - 1 : t - 1);
    const int next = (H >> 1) + (t == half - 1 ? 0 : t + 1);
    const float F[3] = {P.F[0], P.F[1], P.F[2]};
    const int N = P.N;
    int it = 0;
    for (int item = blockIdx.x; item < C.items; item += gridDim.x, ++it) {
        const int s = it % C.stages;
        const uint32_t ph = (it / C.stages) & 1;
        if (!mbar_wait(full + s, ph, C.timeout_ns)) {
            atomicOr(C.err, kDevErrTimeout);
            return;
        }
        const uint32_t* st = reinterpret_cast<const uint32_t*>(ring + s * stage_elems);
        F2 f[Q];
#pragma unroll
        for (int i = 0; i < Q; ++i) {
            const uint32_t* pl = st + i * (pitch >> 1);
            uint32_t w = pl[cur];
            if (L::cx(i) == 1) w = __byte_perm(pl[prev], w, 0x5432);   // nodes pull x - 1
            if (L::cx(i) == -1) w = __byte_perm(w, pl[next], 0x5432);  // nodes pull x + 1
            f[i].v = unpack2<STORE>(w);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);  // the stage may be refilled
        collide2<L, COLL, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
        uint16_t* out = B + item * nx + 2 * t;
#pragma unroll
        for (int i = 0; i < Q; ++i)
            __stcs(reinterpret_cast<unsigned int*>(out + i * N), pack2<STORE>(f[i].v.x, f[i].v.y));
    }
}

// The row-staged kernel handles 16-bit AB steps of fully periodic D3Q19 lattices without
// solids or force fields whose rows are 64..512 nodes, a multiple of 64 (one consumer thread
// per node pair, whole warps); returns 1 for any other case.
template <int STORE, int COLL, bool FORCE>
int go_staged_rows16(const StepParams& P, const void* src, void* dst, cudaStream_t s) {
    const int nx = P.n[0];
    if (!(P.per[0] && P.per[1] && P.per[2]) || nx % 64 != 0 || nx < 64 || nx > 512) return 1;
    const StagedTune t = staged_tune(LBM_D3Q19, 2);
    StagedCfg C;
    C.W = nx;
    C.segs = 1;
    C.items = P.n[1] * P.n[2];
    C.stages = t.stages;
    C.cons_warps = nx / 64;
    C.no_issue = 0;
    C.timeout_ns = 1000000000ull;
    C.err = device_error_ptr();
    if (C.err == nullptr) return int(cudaErrorUnknown);
    const size_t smem = size_t(staged_barrier_bytes(C.stages)) +
                        size_t(C.stages) * 19 * (nx + 16) * sizeof(uint16_t);
    auto kern = k_staged_rows16<STORE, COLL, FORCE>;
    const int threads = 32 * (C.cons_warps + 1);
    static size_t set_smem = 0;
    static int cached_threads = 0, cached_blocks = 0, sms = 0;
    static size_t cached_smem = 0;
    cudaError_t e;
    if (smem > set_smem) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return int(e);
        set_smem = smem;
    }
    if (cached_smem != smem || cached_threads != threads || sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_blocks, kern, threads, smem);
        if (e != cudaSuccess) return int(e);
        cached_smem = smem;
        cached_threads = threads;
    }
    if (cached_blocks < 1) return LBM_E_ARG;
    int grid = cached_blocks * sms;
    if (grid > C.items) grid = C.items;
    kern<<<grid, threads, smem, s>>>(P, C, static_cast<const uint16_t*>(src),
                                     static_cast<uint16_t*>(dst));
    return int(cudaGetLastError());
}

}  // namespace lbm
