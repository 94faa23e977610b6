// State exchange and read-only observables: encode / decode between the canonical float64
// state and the stored buffer, device macroscopic fields, FP64 global moments.
#include <cuda_runtime.h>

#include "codec.cuh"
#include "dispatch.cuh"
#include "lattice.cuh"
#include "params.cuh"

namespace lbm {

namespace {

constexpr int kThreads = 256;

// Stored slot holding population i in the given layout (AA pattern: slot opp(i)).
template <class L>
__device__ __forceinline__ int slot_of(int i, int layout) {
    return layout == LBM_LAYOUT_AA_SWAPPED ? L::opp(i) : i;
}

template <class L, int STORE>
__global__ void k_encode(const double* __restrict__ f64, typename Codec<STORE>::T* buf, int N,
                         int layout) {
    using C = Codec<STORE>;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x) {
        const int n = int(t);
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            double v = f64[(long long)i * N + n];
            if (C::shifted) v -= L::wd(i);
            // same rounding path as pylbm's _encode: float64 -> float32 -> storage type
            buf[(long long)slot_of<L>(i, layout) * N + n] = C::st(float(v));
        }
    }
}

template <class L, int STORE>
__global__ void k_decode(const typename Codec<STORE>::T* __restrict__ buf, double* f64, int N,
                         int layout) {
    using C = Codec<STORE>;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x) {
        const int n = int(t);
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            double v = double(C::ld(buf[(long long)slot_of<L>(i, layout) * N + n]));
            if (C::shifted) v += L::wd(i);
            f64[(long long)i * N + n] = v;
        }
    }
}

// rho and the physical velocity (sum c f - F/2) / rho of the stored post-collision state.
template <class L, int STORE>
__global__ void k_macroscopic(const StepParams P, const typename Codec<STORE>::T* __restrict__ buf,
                              int layout, float* rho_out, float* u_out) {
    using C = Codec<STORE>;
    const int N = P.N;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x) {
        const int n = int(t);
        double s = 0.0, j[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            const double v = double(C::ld(buf[(long long)slot_of<L>(i, layout) * N + n]));
            s += v;
#pragma unroll
            for (int a = 0; a < L::D; ++a) j[a] += double(cc<L>(i, a)) * v;
        }
        const double rho = C::shifted ? 1.0 + s : s;
        rho_out[n] = float(rho);
#pragma unroll
        for (int a = 0; a < L::D; ++a) {
            double F = P.F[a];
            if (P.field) F += double(P.field[(long long)a * N + n]);
            u_out[(long long)a * N + n] = float((j[a] - 0.5 * F) / rho);
        }
    }
}

// Pass 1 of the FP64 moments: one partial (mass, momentum) row per block.
template <class L, int STORE>
__global__ void __launch_bounds__(kThreads)
k_moments_partial(const typename Codec<STORE>::T* __restrict__ buf, int N, int layout,
                  double* __restrict__ partial) {
    using C = Codec<STORE>;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < N;
         t += (long long)gridDim.x * blockDim.x) {
        const int n = int(t);
#pragma unroll
        for (int i = 0; i < L::Q; ++i) {
            const double v = double(C::ld(buf[(long long)slot_of<L>(i, layout) * N + n]));
            acc[0] += v;
#pragma unroll
            for (int a = 0; a < L::D; ++a) acc[1 + a] += double(cc<L>(i, a)) * v;
        }
    }
    __shared__ double red[kThreads / 32][4];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = warp_sum(acc[k]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x < 4) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
        partial[blockIdx.x * 4 + threadIdx.x] = s;
    }
}

// Pass 2: one block sums the partial rows in a fixed order (bitwise reproducible).
template <class L, bool SHIFTED>
__global__ void __launch_bounds__(kThreads)
k_moments_final(const double* __restrict__ partial, int rows, int N, double* out) {
    __shared__ double red[kThreads / 32][4];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int r = threadIdx.x; r < rows; r += kThreads)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += partial[r * 4 + k];
#pragma unroll
    for (int k = 0; k < 4; ++k) acc[k] = warp_sum(acc[k]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 4; ++k) red[warp][k] = acc[k];
    __syncthreads();
    if (threadIdx.x <= L::D) {
        double s = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
        // shifted storages hold f - w_i: sum w_i = 1 per node, sum w_i c_i = 0
        if (SHIFTED && threadIdx.x == 0) s += double(N);
        out[threadIdx.x] = s;
    }
}

int grid_for(long long work) {
    long long g = (work + kThreads - 1) / kThreads;
    if (g > kHelperGridMax) g = kHelperGridMax;
    return int(g < 1 ? 1 : g);
}

template <class L, int STORE>
int moments_impl(const void* f, int N, int layout, double* out, double* scratch, int rows,
                 cudaStream_t s) {
    using T = typename Codec<STORE>::T;
    k_moments_partial<L, STORE><<<rows, kThreads, 0, s>>>(static_cast<const T*>(f), N, layout,
                                                         scratch);
    k_moments_final<L, Codec<STORE>::shifted><<<1, kThreads, 0, s>>>(scratch, rows, N, out);
    return int(cudaGetLastError());
}

template <class L>
int moments_storage(const LbmDesc& d, const void* f, int layout, double* out, double* scratch,
                    int rows, cudaStream_t s) {
    const int N = make_params(d).N;
    switch (d.storage) {
        case LBM_STORE_F32: return moments_impl<L, LBM_STORE_F32>(f, N, layout, out, scratch, rows, s);
        case LBM_STORE_F16: return moments_impl<L, LBM_STORE_F16>(f, N, layout, out, scratch, rows, s);
        case LBM_STORE_BF16:
            return moments_impl<L, LBM_STORE_BF16>(f, N, layout, out, scratch, rows, s);
        case LBM_STORE_F32_SHIFTED:
            return moments_impl<L, LBM_STORE_F32_SHIFTED>(f, N, layout, out, scratch, rows, s);
    }
    return LBM_E_STORAGE;
}

// Dispatch helper: calls fn.template operator()<L, STORE>() for the descriptor's types.
template <class Fn>
int with_types(const LbmDesc& d, Fn&& fn) {
    auto by_store = [&](auto lat) -> int {
        using L = decltype(lat);
        switch (d.storage) {
            case LBM_STORE_F32: return fn.template operator()<L, LBM_STORE_F32>();
            case LBM_STORE_F16: return fn.template operator()<L, LBM_STORE_F16>();
            case LBM_STORE_BF16: return fn.template operator()<L, LBM_STORE_BF16>();
            case LBM_STORE_F32_SHIFTED: return fn.template operator()<L, LBM_STORE_F32_SHIFTED>();
        }
        return LBM_E_STORAGE;
    };
    return d.lattice == LBM_D2Q9 ? by_store(D2Q9{}) : by_store(D3Q19{});
}

}  // namespace

int launch_encode(const LbmDesc& d, const double* f64, void* buf, int layout, cudaStream_t s) {
    const int N = make_params(d).N;
    return with_types(d, [&]<class L, int STORE>() {
        using T = typename Codec<STORE>::T;
        k_encode<L, STORE><<<grid_for(N), kThreads, 0, s>>>(f64, static_cast<T*>(buf), N, layout);
        return int(cudaGetLastError());
    });
}

int launch_decode(const LbmDesc& d, const void* buf, int layout, double* f64, cudaStream_t s) {
    const int N = make_params(d).N;
    return with_types(d, [&]<class L, int STORE>() {
        using T = typename Codec<STORE>::T;
        k_decode<L, STORE><<<grid_for(N), kThreads, 0, s>>>(static_cast<const T*>(buf), f64, N,
                                                           layout);
        return int(cudaGetLastError());
    });
}

int launch_macroscopic(const LbmDesc& d, const void* f, int layout, float* rho, float* u,
                       cudaStream_t s) {
    const StepParams P = make_params(d);
    return with_types(d, [&]<class L, int STORE>() {
        using T = typename Codec<STORE>::T;
        k_macroscopic<L, STORE><<<grid_for(P.N), kThreads, 0, s>>>(P, static_cast<const T*>(f),
                                                                  layout, rho, u);
        return int(cudaGetLastError());
    });
}

int moments_rows(int N) { return grid_for(N); }

// The two moment passes with caller-provided scratch of at least 4 * rows doubles.
int launch_moments_into(const LbmDesc& d, const void* f, int layout, double* out,
                        double* scratch, int rows, cudaStream_t s) {
    return d.lattice == LBM_D2Q9 ? moments_storage<D2Q9>(d, f, layout, out, scratch, rows, s)
                                 : moments_storage<D3Q19>(d, f, layout, out, scratch, rows, s);
}

// The partial rows live in stream-ordered scratch from cudaMallocAsync, released on the
// same stream after pass 2 has consumed them.
int launch_moments(const LbmDesc& d, const void* f, int layout, double* out, cudaStream_t s) {
    const int N = make_params(d).N;
    const int rows = grid_for(N);
    double* scratch = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&scratch),
                                    sizeof(double) * 4 * rows, s);
    if (e != cudaSuccess) return int(e);
    const int rc = d.lattice == LBM_D2Q9
                       ? moments_storage<D2Q9>(d, f, layout, out, scratch, rows, s)
                       : moments_storage<D3Q19>(d, f, layout, out, scratch, rows, s);
    e = cudaFreeAsync(scratch, s);
    if (rc != 0) return rc;
    return int(e);
}

}  // namespace lbm
