// lbm_moments_f64_noalloc: the FP64 mass / momentum sums without any device allocation.
//
// lbm_moments_f64 takes its partial-sum scratch from cudaMallocAsync on every call. Some
// callers cannot let a library allocate: applications that hand all device memory to their own
// pool allocator and forbid allocations behind its back, and long-running loops that must not
// risk an allocation stall or an out-of-memory failure halfway through a run. This entry point
// runs the same two reduction passes with the partial sums in a fixed array that lives in the
// library's device image instead.
//
// The array holds kMaxRows rows of 4 doubles (2368 rows, 75,776 bytes). Each device that loads
// the library keeps its own copy until the process exits. The reduction uses one row per block
// of the first pass and never more than kMaxRows for any problem the library accepts; a
// problem that would need more is refused with LBM_E_SIZE.
//
// In host code the name g_partials only stands for the array; it is not a device address. The
// first call on each device, with that device current, looks the address up with
// cudaGetSymbolAddress and keeps it together with the id of the CUDA context it belongs to;
// a later call in another context of that device (after a device reset, say) looks it up
// again. Make the first call on a device before any stream capture. Every call shares the one
// array and leaves its partial sums behind. Pass 1 writes every row that pass 2 reads, so
// nothing has to be cleared between calls, but calls that overlap on the GPU (for example on
// two streams) race on the array and must be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "../../include/pylbm_b200.h"
#include "dispatch.cuh"

namespace {

constexpr int kMaxRows = lbm::kHelperGridMax;  // 2368 rows of 4 doubles
static_assert(kMaxRows == 2368, "the documented size of the fixed array");
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxRows * 4];

// Per device: the address of g_partials and the id of the context it was looked up in.
// The address is stored before the id (release) and read after it (acquire), so a caller
// that sees a matching id also sees that context's address.
struct Slot {
    std::atomic<double*> addr{nullptr};
    std::atomic<unsigned long long> ctx_id{0};
};
Slot g_slots[kMaxDevices];

// Unique id of the current context (0 when there is none yet). The two driver functions are
// fetched through the runtime, so the library does not link the driver library directly and
// still loads (for its argument checks) on machines without one.
unsigned long long current_ctx_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static std::atomic<GetCurrent> get_current{nullptr};
    static std::atomic<GetId> get_id{nullptr};
    GetCurrent gc = get_current.load(std::memory_order_acquire);
    GetId gi = get_id.load(std::memory_order_acquire);
    if (gc == nullptr || gi == nullptr) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) !=
                cudaSuccess || qa != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qb != cudaDriverEntryPointSuccess)
            return 0;
        gc = reinterpret_cast<GetCurrent>(a);
        gi = reinterpret_cast<GetId>(b);
        get_current.store(gc, std::memory_order_release);
        get_id.store(gi, std::memory_order_release);
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (gc(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
    if (gi(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of g_partials in the current context of the current device.
int partials_address(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return int(e);
    if (dev < 0 || dev >= kMaxDevices) return LBM_E_ARG;
    Slot& slot = g_slots[dev];
    unsigned long long id = current_ctx_id();
    if (id != 0 && slot.ctx_id.load(std::memory_order_acquire) == id) {
        *out = slot.addr.load(std::memory_order_relaxed);
        return LBM_OK;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);  // makes the device's context current if needed
    if (e != cudaSuccess) return int(e);
    id = current_ctx_id();
    slot.addr.store(static_cast<double*>(p), std::memory_order_relaxed);
    slot.ctx_id.store(id, std::memory_order_release);
    *out = static_cast<double*>(p);
    return LBM_OK;
}

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace

extern "C" int lbm_moments_f64_noalloc(const LbmDesc* d, const void* f, int layout,
                                       double* out, uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if (f == nullptr || out == nullptr) return LBM_E_NULL;
    const uintptr_t es = (d->storage == LBM_STORE_F16 || d->storage == LBM_STORE_BF16) ? 2 : 4;
    if (!aligned(f, es) || !aligned(out, 8)) return LBM_E_ALIGN;
    if (layout != LBM_LAYOUT_NATURAL && layout != LBM_LAYOUT_AA_SWAPPED) return LBM_E_ARG;
    const int N = d->nx * d->ny * (d->lattice == LBM_D2Q9 ? 1 : d->nz);
    const int rows = lbm::moments_rows(N);
    if (rows > kMaxRows) return LBM_E_SIZE;
    double* scratch = nullptr;
    if ((rc = partials_address(&scratch))) return rc;
    return lbm::launch_moments_into(*d, f, layout, out, scratch, rows,
                                    reinterpret_cast<cudaStream_t>(stream));
}
