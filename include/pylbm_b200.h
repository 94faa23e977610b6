/*
 * pylbm_b200 -- C ABI of the B200 (sm_100a) fused lattice-Boltzmann stream-collide library.
 *
 * Every entry point takes plain pointers, sizes and a CUDA stream handle (cast to uint64_t);
 * no torch or C++ types cross this boundary. Device buffers are owned by the caller and are
 * never freed by the library. Launches are asynchronous on the given stream.
 *
 * Return value of every int-returning call: 0 on success, a negative LBM_E_* code for an
 * invalid argument (nothing was launched), or a positive cudaError_t value when the CUDA
 * runtime reported an error. lbm_error_string() turns any of them into text.
 *
 * Layouts (identical to pylbm's):
 *   population buffer: structure of arrays, element (i, n) at index i * N + n,
 *   n = x + nx * (y + ny * z), N = nx * ny * nz, q planes (9 for D2Q9, 19 for D3Q19).
 *   Velocity orders, weights and opposite tables follow pylbm's lattice.py:
 *     D2Q9  0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE
 *     D3Q19 0 rest, then opposite pairs adjacent: (1,2) (3,4) ... (17,18)
 *   The stored value is f (LBM_STORE_F32) or f - w_i (the three shifted storages).
 *   AA-pattern buffers between step pairs hold population i in slot opp(i).
 */
#ifndef PYLBM_B200_H
#define PYLBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 2

/* lattices */
#define LBM_D2Q9 0
#define LBM_D3Q19 1
/* collision operators */
#define LBM_BGK 0
#define LBM_TRT 1
#define LBM_MRT 2 /* D2Q9: Lallemand-Luo basis (pylbm); D3Q19: d'Humieres et al. (2002) basis */
#define LBM_STREAM_ONLY 3 /* debug: streaming and boundaries only, no collision */
/* storage formats; arithmetic is fp32 in every case */
#define LBM_STORE_F32 0         /* f in fp32, unshifted arithmetic (pylbm's own fp32 scheme) */
#define LBM_STORE_F16 1         /* f - w_i in fp16, shifted arithmetic */
#define LBM_STORE_BF16 2        /* f - w_i in bf16, shifted arithmetic */
#define LBM_STORE_F32_SHIFTED 3 /* f - w_i in fp32, shifted arithmetic */
/* streaming patterns */
#define LBM_PATTERN_AB 0      /* pull, reads src, writes dst (src != dst) */
#define LBM_PATTERN_AA_ODD 1  /* in place: reads swapped layout, writes natural layout */
#define LBM_PATTERN_AA_EVEN 2 /* in place: reads natural layout, writes swapped layout */
/* buffer layouts for the read-only helpers */
#define LBM_LAYOUT_NATURAL 0
#define LBM_LAYOUT_AA_SWAPPED 1

/* error codes (negative; positive values are cudaError_t) */
#define LBM_OK 0
#define LBM_E_NULL -1        /* a required pointer is NULL */
#define LBM_E_LATTICE -2     /* unknown lattice id */
#define LBM_E_COLLISION -3   /* unknown collision operator */
#define LBM_E_STORAGE -4     /* unknown storage id */
#define LBM_E_PATTERN -5     /* unknown pattern id */
#define LBM_E_SHAPE -6       /* a dimension < 1, or nz != 1 for D2Q9 */
#define LBM_E_INDEX -7       /* q * N does not fit in int32 (pylbm's fused-kernel limit) */
#define LBM_E_RATE -8        /* a relaxation rate or force is not finite, or rate outside (0, 2) */
#define LBM_E_LID -9         /* moving lid requested on a periodic last axis */
#define LBM_E_ALIGN -10      /* a device pointer is not aligned to its element size (16 B for buffers) */
#define LBM_E_ALIAS -11      /* AB pattern with src == dst, or AA pattern with src != dst */
#define LBM_E_STEPS -12      /* negative step count, or odd count for the AA pattern */
#define LBM_E_TIMEOUT -13    /* a bounded device-side wait gave up (error flag set by the kernel) */
#define LBM_E_HANDLE -14     /* unknown or destroyed handle */
#define LBM_E_ARG -15        /* any other invalid argument */
#define LBM_E_SIZE -16       /* problem larger than a fixed capacity */
#define LBM_E_INOUT -17      /* inlet / outlet without D2Q9, x walls and the two-buffer pull */

/* Problem descriptor: the compile-time #defines and runtime scalars of pylbm's fused kernel
 * (backends/cupy_backend.py:51-70 header, backends/_fused.py:129-136 scalar_args) as one POD.
 * Rates follow codegen.py:437-445 runtime_rates: BGK r0 = 1/tau; TRT r0 = s+, r1 = s-;
 * MRT r0 = s_nu, r1 = s_e, r2 = s_eps, r3 = s_q. */
typedef struct LbmDesc {
    int32_t lattice;
    int32_t collision;
    int32_t storage;
    int32_t periodic_mask; /* bit a set: axis a (0 = x, 1 = y, 2 = z) is periodic, else walls */
    int32_t nx, ny, nz;    /* nz = 1 for D2Q9 */
    float ulid;            /* lid speed: top wall of the last axis moving in +x; 0 = no lid */
    float fx, fy, fz;      /* uniform Guo body force (fz ignored in 2D) */
    float r0, r1, r2, r3;  /* relaxation rates, see above */
    /* optional extensions beyond pylbm's fused kernel (NULL = off) */
    const uint32_t* solid_bits; /* 1 bit per node: bit (n & 31) of word (n >> 5); solid nodes
                                   act as stationary half-way bounce-back obstacles */
    const float* force_field;   /* per-node force added to (fx, fy, fz): layout (d, N) fp32 */
    double* mx_force;           /* momentum-exchange force on the solids, added (not stored)
                                   into mx_force[0..d-1] by each step that writes a state */
    int64_t mx_stride;          /* doubles between the slots of consecutive steps in
                                   lbm_advance (0 = every step adds into the same slot) */
    int32_t flags;              /* LBM_FLAG_* bits, 0 by default */
    int32_t outlet;             /* 1: pressure outlet on the right boundary (pylbm's
                                   Problem.outlet, core.py:130-148); D2Q9, x walls, AB only */
    const float* inlet_u;       /* velocity inlet on the left wall (Problem.inlet,
                                   core.py:67-78,116-117): u_x per row y, ny floats on the
                                   device; D2Q9, x walls, AB only */
} LbmDesc;

/* descriptor flags */
#define LBM_FLAG_GENERIC 1 /* always use the one-node-per-thread kernel (for A/B testing) */
#define LBM_FLAG_STAGED 2  /* use the TMA-staged kernels instead of the register ones (D2Q9 and
                              D3Q19 row segments; 16-bit D3Q19 AB on fully periodic rows of
                              64..512 nodes: whole staged rows; D3Q19 MRT has no staged form
                              and ignores it); slower, kept as an option */

/* Library identification. */
int lbm_abi_version(void);
const char* lbm_error_string(int code);

/* Host-only: the lattice tables compiled into the kernels (c as q rows of 3, w, opp), so a
 * caller can check them against pylbm's lattice.py:49-67 without a GPU. */
int lbm_lattice_info(int lattice, int* q, int* dim, int* c, double* w, int* opp);

/* Host-only validation of a descriptor (no GPU needed). Same checks as the launch paths:
 * pylbm's capability gate backends/_fused.py:54-66 (q*N < 2^31) and problem.py:44-61. */
int lbm_validate(const LbmDesc* d);

/* One fused stream-collide launch of the given pattern.
 * Replaces FusedSolver._launch (backends/_fused.py:112-114, cupy_backend.py:101-103):
 * 'ab' reads src and writes dst; 'aa-odd' / 'aa-even' update src in place (dst == src). */
int lbm_launch(const LbmDesc* d, const void* src, void* dst, int pattern, uint64_t stream);

/* Advance nsteps time steps. Replaces FusedSolver._advance (backends/_fused.py:116-124).
 * aa = 0: pull two-buffer; step k reads (k even ? a : b) and writes the other buffer, so the
 *         result is in a when nsteps is even and in b when it is odd.
 * aa = 1: AA in place on a (b ignored); nsteps must be even (odd + even launch per pair). */
int lbm_advance(const LbmDesc* d, void* a, void* b, int aa, int nsteps, uint64_t stream);

/* FP64 global sums of a stored state: out[0] = sum rho (mass), out[1..d] = sum c f
 * (momentum), written to DEVICE memory out[0..d]. Deterministic two-pass reduction.
 * No pylbm counterpart as a kernel; the host equivalent is core.py:255-266 summed. */
int lbm_moments_f64(const LbmDesc* d, const void* f, int layout, double* out,
                    uint64_t stream);

/* The same sums without allocating: for callers that cannot let a library allocate device
 * memory (an application whose own pool owns all of it, or a loop that must not risk an
 * allocation stall or failure mid-run). No counterpart in pylbm. The partial sums live in a
 * fixed 75,776-byte array in the library's device image (2368 rows; larger needs are refused
 * with LBM_E_SIZE), one copy per device until exit. The first call on a device (and the first
 * in a new context of it, e.g. after a device reset) looks up that array's address and should
 * come before any stream capture. All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int lbm_moments_f64_noalloc(const LbmDesc* d, const void* f, int layout, double* out,
                            uint64_t stream);

/* Device macroscopic fields from a stored state: rho[N], u[d * N] (fp32), with the physical
 * velocity u = (sum c f - F/2) / rho of pylbm's core.macroscopic (core.py:255-266). */
int lbm_macroscopic(const LbmDesc* d, const void* f, int layout, float* rho, float* u,
                    uint64_t stream);

/* Canonical float64 populations (q, N) <-> stored buffer, on the device.
 * Replaces FusedSolver._encode / populations (backends/_fused.py:83-103): subtracts or adds
 * w_i for shifted storages and applies the AA slot swap when layout = LBM_LAYOUT_AA_SWAPPED. */
int lbm_encode_f64(const LbmDesc* d, const double* f64, void* buf, int layout,
                   uint64_t stream);
int lbm_decode_f64(const LbmDesc* d, const void* buf, int layout, double* f64,
                   uint64_t stream);

/* Batches of independent D2Q9 lattices of uneven sizes (no pylbm counterpart: pylbm steps
 * one lattice per solver). All lattices share collision and storage; each has its own shape,
 * walls, lid speed and rates; nx must be a multiple of the 16-byte vector (4 fp32 / 8 x
 * 16-bit). Lattice l occupies elements [offset_l, offset_l + 9 nx_l ny_l) of the two caller
 * buffers, in the order given. One kernel launch advances every lattice by one step. */
typedef struct LbmBatch LbmBatch;
int lbm_batch_create(const LbmDesc* lattices, int count, LbmBatch** out);
int lbm_batch_destroy(LbmBatch* b);
int lbm_batch_info(const LbmBatch* b, int64_t* elements, int64_t* nodes, int* items);
int lbm_batch_offsets(const LbmBatch* b, int64_t* offsets);
/* launch shape, chosen by the autotuner: threads per block (64/128/256) and resident blocks
 * per SM (1..64: a persistent grid whose warps stride over the work items; 0: one work item
 * per warp) */
int lbm_batch_set_launch(LbmBatch* b, int block, int blocks_per_sm);
int lbm_batch_get_launch(const LbmBatch* b, int* block, int* blocks_per_sm);
/* nsteps pull steps, ping-pong a -> b -> a ...: the result is in a when nsteps is even */
int lbm_batch_step(LbmBatch* b, void* a, void* bb, int nsteps, uint64_t stream);
/* the same nsteps launches replayed from one CUDA graph, captured on first use for these
 * buffers, step count and launch shape, and cached in the batch */
int lbm_batch_graph_launch(LbmBatch* b, void* a, void* bb, int nsteps, uint64_t stream);

/* Adjoint of the D2Q9 BGK step (Guo forcing with LbmDesc.force_field, walls, periodic axes,
 * solids; shifted storages), for the gradient of a momentum-exchange objective with respect
 * to the per-node force field. No pylbm counterpart (pylbm computes the momentum-exchange
 * force, karman.py:45-53,88-96, but has no gradients).
 * lbm_forward_record: one AB step src -> dst that also writes the rho and u its collision
 *   used, rho_u = 3 planes of N floats (rho, ux, uy): the recomputation pass of checkpointing.
 * lbm_adjoint_step: one reverse step. lambda_{t+1} = objw * dPhi/df + P^T mu_in (mu_in NULL
 *   for the last step), mu_out = (dC/dg)^T lambda_{t+1}, grad (2 N doubles) +=
 *   (dC/dF)^T lambda_{t+1}; rho_u is the record of the forward step t -> t+1; objw is the
 *   weight of Phi(f_{t+1}) = x momentum-exchange force on the solids in the objective. */
int lbm_forward_record(const LbmDesc* d, const void* src, void* dst, float* rho_u,
                       uint64_t stream);
int lbm_adjoint_step(const LbmDesc* d, const float* rho_u, const float* mu_in, float* mu_out,
                     double* grad, double objw, uint64_t stream);

/* Tuning of the TMA-staged kernels (D3Q19 always; D2Q9 with LBM_FLAG_STAGED), per lattice and
 * stored element size (2 or 4 bytes), process-wide: nodes per row segment (multiple of 8),
 * shared-memory ring depth (2..8) and consumer warps (1..8). No pylbm counterpart (pylbm
 * launches one fixed block shape, _fused.py:26-31); used by the autotuner. */
int lbm_set_staged_config(int lattice, int elem_bytes, int width, int stages, int warps);
int lbm_get_staged_config(int lattice, int elem_bytes, int* width, int* stages, int* warps);

/* Synchronise the current device and report its device error word: LBM_OK, or LBM_E_TIMEOUT
 * when a kernel's bounded wait gave up since the last clear (clear != 0 resets the word). */
int lbm_device_error(int clear);

/* Failure-detection self test (D3Q19 descriptor, any 16-byte aligned buffer that is left
 * untouched): launches the staged kernel with its copy producer disabled, so every consumer
 * wait runs out after timeout_ns (0 < timeout_ns <= 10 s); lbm_device_error() then reports
 * LBM_E_TIMEOUT and the context stays usable. */
int lbm_selftest_wait_timeout(const LbmDesc* d, void* buf, uint64_t timeout_ns,
                              uint64_t stream);

#ifdef __cplusplus
}
#endif

#endif /* PYLBM_B200_H */
