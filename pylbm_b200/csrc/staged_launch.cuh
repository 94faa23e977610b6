// Host-side launch of the TMA-staged kernels, and the lattice-generic AA-even vector kernel.
#pragma once

#include <cuda_runtime.h>

#include "dispatch.cuh"
#include "step_staged.cuh"
#include "vec.cuh"

namespace lbm {

template <class L, int STORE, int COLL, bool FORCE, int PATTERN>
int go_staged(const StepParams& P, const void* src, void* dst, cudaStream_t s,
              int no_issue = 0, unsigned long long timeout_ns = 1000000000ull) {
    using E = typename VT<STORE>::E;
    constexpr int V = VT<STORE>::V;
    constexpr int H = V;
    const StagedTune t = staged_tune(L::D == 2 ? LBM_D2Q9 : LBM_D3Q19, int(sizeof(E)));
    StagedCfg C;
    const int nx_r = ((P.n[0] + V - 1) / V) * V;
    C.W = ((t.width + V - 1) / V) * V;
    if (C.W > nx_r) C.W = nx_r;
    C.segs = (P.n[0] + C.W - 1) / C.W;
    C.items = C.segs * P.n[1] * P.n[2];
    C.stages = t.stages;
    C.cons_warps = t.warps;
    C.no_issue = no_issue;
    C.timeout_ns = timeout_ns;
    C.err = device_error_ptr();
    if (C.err == nullptr) return int(cudaErrorUnknown);
    const size_t smem = size_t(staged_barrier_bytes(C.stages)) +
                        size_t(C.stages) * L::Q * (C.W + 2 * H) * sizeof(E);
    auto kern = k_staged<L, STORE, COLL, FORCE, PATTERN>;
    const int threads = 32 * (C.cons_warps + 1);
    // cached per instantiation: shared-memory opt-in and resident CTAs per SM
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
    kern<<<grid, threads, smem, s>>>(P, C, static_cast<const E*>(src), static_cast<E*>(dst));
    return int(cudaGetLastError());
}

// AA even step: read A[i, x], collide, write A[opp(i), x]; purely node-local, so one aligned
// 16-byte vector per plane and lane.
template <class L, int STORE, int COLL, bool FORCE>
__global__ void __launch_bounds__(128) k_aa_even(const StepParams P, void* Av) {
    using E = typename VT<STORE>::E;
    using T = VT<STORE>;
    constexpr int V = T::V;
    constexpr int Q = L::Q;
    E* A = static_cast<E*>(Av);
    const int n0 = (blockIdx.x * blockDim.x + threadIdx.x) * V;
    if (n0 >= P.N) return;
    uint4 v[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) v[i] = ld_plain(A + i * P.N + n0);
    const float F[3] = {P.F[0], P.F[1], P.F[2]};
    if constexpr (COLL == LBM_MRT) {  // one copy of the moment transform (step_rows3d.cuh)
#pragma unroll 1
        for (int k = 0; k < V; ++k) {
            float f[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] = T::f(elem<V>(v[i], 0));
            collide<L, COLL, Codec<STORE>::shifted, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < Q; ++i) v[i] = shift_down<V>(v[i], T::b(f[i]));
        }
    } else if constexpr (V == 4) {
#pragma unroll
        for (int k = 0; k < V; ++k) {
            float f[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i] = T::f(elem<V>(v[i], k));
            collide<L, COLL, Codec<STORE>::shifted, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < Q; ++i) put<V>(v[i], k, T::b(f[i]));
        }
    } else {
        // 16-bit: the two nodes of a word collided together with packed f32x2 instructions
        // (bit-for-bit the one-node result). No register cap: the kernel takes 255 registers
        // (2 blocks per SM) and keeps 19 loads in flight per thread; capped at 128 it measured
        // slower (D3Q19 256^3 TRT fp16 AA pair 0.861 -> 0.707 of copy, one-node 0.851 -> 0.813),
        // at 168 (3 blocks) 0.879 -> 0.869, and 8-byte lanes (4 nodes) gained nothing
#pragma unroll
        for (int jw = 0; jw < 4; ++jw) {
            F2 f[Q];
#pragma unroll
            for (int i = 0; i < Q; ++i) f[i].v = unpack2<STORE>(word(v[i], jw));
            collide2<L, COLL, FORCE>(f, F, P.r0, P.r1, P.r2, P.r3);
#pragma unroll
            for (int i = 0; i < Q; ++i) set_word(v[i], jw, pack2<STORE>(f[i].v.x, f[i].v.y));
        }
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) st_cs(A + L::opp(i) * P.N + n0, v[i]);
}

template <class L, int STORE, int COLL, bool FORCE>
int go_aa_even(const StepParams& P, void* dst, cudaStream_t s) {
    constexpr int V = VT<STORE>::V;
    const int threads = P.N / V;
    k_aa_even<L, STORE, COLL, FORCE><<<(threads + 127) / 128, 128, 0, s>>>(P, dst);
    return int(cudaGetLastError());
}

}  // namespace lbm
