// Launcher for pylbm's own CUDA C kernel (backends/cuda/lbm.cu) -- test infrastructure only.
//
// The kernel source is compiled from the reference tree where it lies (LBM_REF_CU is its
// path), preceded by a configuration header of #defines (Q, D, lattice tables, PER_*, LID,
// FORCE, COLL, STORAGE, PATTERN, BLOCK_X) written by oracle/build_ref.py in the role of
// pylbm's kernel_source() (cupy_backend.py:51-70). The launch mirrors CupyFused._compile /
// _launch (cupy_backend.py:95-103): grid (ceil(nx / BLOCK_X), ny, nz), block (BLOCK_X, 1, 1),
// int32 sizes and float32 scalars.
#include <cuda_runtime.h>

#include LBM_REF_CU

extern "C" int ref_lbm_launch(const void* A, void* B, int nx, int ny, int nz, int N,
                              float ulid, float fx, float fy, float fz, float r0, float r1,
                              float r2, float r3, unsigned long long stream) {
    const dim3 grid((nx + BLOCK_X - 1) / BLOCK_X, ny, nz);
    lbm_kernel<<<grid, BLOCK_X, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const store_t*>(A), static_cast<store_t*>(B), nx, ny, nz, N, ulid, fx, fy,
        fz, r0, r1, r2, r3);
    return int(cudaGetLastError());
}

extern "C" int ref_lbm_config(int* q, int* pattern, int* storage, int* coll) {
    *q = Q;
    *pattern = PATTERN;
    *storage = STORAGE;
    *coll = COLL;
    return 0;
}
