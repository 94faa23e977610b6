// The device-side error word: kernels whose bounded waits give up record an error code here
// (atomicOr of LBM_DEVERR_* bits) and return instead of spinning on.
#include <cuda_runtime.h>

#include "dispatch.cuh"

namespace lbm {

namespace {
__device__ unsigned int g_device_error = 0u;
constexpr int kMaxDevices = 64;
unsigned int* g_ptr[kMaxDevices] = {};
}  // namespace

unsigned int* device_error_ptr() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    if (g_ptr[dev] == nullptr) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_device_error) != cudaSuccess) return nullptr;
        g_ptr[dev] = static_cast<unsigned int*>(p);
    }
    return g_ptr[dev];
}

int read_device_error(int clear, unsigned int* bits) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return int(e);
    unsigned int v = 0;
    e = cudaMemcpyFromSymbol(&v, g_device_error, sizeof(v));
    if (e != cudaSuccess) return int(e);
    if (clear && v) {
        const unsigned int zero = 0;
        e = cudaMemcpyToSymbol(g_device_error, &zero, sizeof(zero));
        if (e != cudaSuccess) return int(e);
    }
    *bits = v;
    return 0;
}

}  // namespace lbm
