// Host-side launchers shared between translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/pylbm_b200.h"
#include "params.cuh"

namespace lbm {

// True when the step needs the Guo source terms.
inline bool needs_force(const LbmDesc& d) {
    return d.fx != 0.0f || d.fy != 0.0f || (d.lattice == LBM_D3Q19 && d.fz != 0.0f) ||
           d.force_field != nullptr;
}

inline int block_x_for(int nx) {
    for (int b : {128, 64, 32})
        if (nx % b == 0) return b;
    return 128;
}

// One launch of the generic kernel (step_generic_*.cu). Arguments are validated.
int launch_generic_d2q9(const LbmDesc& d, const void* src, void* dst, int pattern,
                        cudaStream_t s);
int launch_generic_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern,
                         cudaStream_t s);

// Specialised kernels; each returns 1 when it does not handle the case (the caller then
// uses the generic kernel), else 0 or a cudaError_t.
int launch_fast_d2q9(const LbmDesc& d, const void* src, void* dst, int pattern,
                     cudaStream_t s);
int launch_fast_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern,
                      cudaStream_t s);
// D3Q19 MRT on the register row kernels (step_d3q19_mrt.cu), for descriptors that
// launch_fast_d3q19 accepts.
int launch_mrt_d3q19(const LbmDesc& d, const void* src, void* dst, int pattern, cudaStream_t s);

// One lattice of a batch (device table entry, batched.cu / step_d2q9.cu).
struct BatchLattice {
    long long base;     // element offset of the lattice's plane 0 in the batch buffers
    int nx, ny;
    int periodic_mask;
    int item0;          // first warp work item of the lattice
    int segs;           // V-node vectors per row (a work item is 32 consecutive vectors)
    int y0, xv0;        // per-item copies: row and vector offset of the item's first vector
    float ulid, r0, r1, r2, r3;
};

// One step of every lattice of a batch (D2Q9 pull, two buffers). item_tab[k] holds the
// parameters of the lattice of work item k; persist selects the grid-stride kernel (grid
// smaller than the item count) over the one-item-per-warp kernel (grid covering every item).
int launch_batch_d2q9(int collision, int storage, const BatchLattice* item_tab, int items,
                      const void* src, void* dst, int grid, int block, bool persist,
                      cudaStream_t s);

// Per-launch configuration of the TMA-staged kernels (see lbm_set_staged_config).
struct StagedTune {
    int width;   // nodes per row segment
    int stages;  // ring depth
    int warps;   // consumer warps
};

// Process-wide tuning table (abi.cu), by lattice and bytes per stored element.
StagedTune staged_tune(int lattice, int elem_bytes);

// Device error word (errors.cu): its device address on the current device, and a read that
// synchronises the device first.
unsigned int* device_error_ptr();
int read_device_error(int clear, unsigned int* bits);

// Staged-kernel self test (step_d3q19.cu): a launch whose producer issues no copy, so every
// consumer wait runs out after timeout_ns and records the timeout in the device error word.
int launch_staged_timeout_probe(const LbmDesc& d, void* buf, unsigned long long timeout_ns,
                                cudaStream_t s);

// Helpers (helpers.cu)
int launch_encode(const LbmDesc& d, const double* f64, void* buf, int layout, cudaStream_t s);
int launch_decode(const LbmDesc& d, const void* buf, int layout, double* f64, cudaStream_t s);
int launch_macroscopic(const LbmDesc& d, const void* f, int layout, float* rho, float* u,
                       cudaStream_t s);
int launch_moments(const LbmDesc& d, const void* f, int layout, double* out, cudaStream_t s);
// Grid cap of the node-parallel helper kernels (encode, decode, macroscopic, the moment
// reduction's first pass): 16 blocks per SM of the 148. It is also the most rows of partial
// sums the moment reduction ever uses, which bounds the allocation-free entry point's array.
constexpr int kHelperGridMax = 148 * 16;
// Rows of partial sums the moment reduction uses for N nodes (at most kHelperGridMax), and
// the reduction into caller-provided scratch of 4 * rows doubles.
int moments_rows(int N);
int launch_moments_into(const LbmDesc& d, const void* f, int layout, double* out,
                        double* scratch, int rows, cudaStream_t s);

}  // namespace lbm
