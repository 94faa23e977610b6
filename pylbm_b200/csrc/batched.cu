// Batches of independent D2Q9 lattices of uneven sizes advanced by one launch per step, and
// CUDA graphs of such steps.
//
// A batch owns a device table (the parameters of every work item's lattice) and its cached
// graph executables; the population buffers are the caller's. Lattice l occupies elements
// [base_l, base_l + 9 N_l) of each buffer, lattices back to back in the order given, so
// every lattice's planes start 16-byte aligned (nx is a multiple of the 16-byte vector).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/pylbm_b200.h"
#include "dispatch.cuh"
#include "lattice.cuh"

struct LbmBatch {
    int count = 0;
    int collision = 0;
    int storage = 0;
    int items = 0;
    long long elements = 0;
    long long nodes = 0;
    std::vector<long long> bases;
    lbm::BatchLattice* item_tab = nullptr;  // device, the lattice of every work item
    int block = 256;
    int blocks_per_sm = 8;
    int sms = 0;
    // cached graph: nsteps launches on fixed buffers with a fixed launch shape
    cudaGraphExec_t exec = nullptr;
    const void* g_a = nullptr;
    const void* g_b = nullptr;
    int g_steps = 0, g_block = 0, g_grid = 0;
};

namespace {

int vec_elems(int storage) {
    return (storage == LBM_STORE_F16 || storage == LBM_STORE_BF16) ? 8 : 4;
}

// blocks_per_sm = 0: one work item per warp (no grid-stride loop)
int grid_of(const LbmBatch& b) {
    const long long need = ((long long)b.items * 32 + b.block - 1) / b.block;
    long long g = b.blocks_per_sm > 0 ? (long long)b.blocks_per_sm * b.sms : need;
    if (g > need) g = need;
    return int(g < 1 ? 1 : g);
}

int launch_steps(LbmBatch* b, void* a, void* bb, int nsteps, cudaStream_t s) {
    const int grid = grid_of(*b);
    for (int k = 0; k < nsteps; ++k) {
        const void* src = (k & 1) ? bb : a;
        void* dst = (k & 1) ? a : bb;
        const int rc = lbm::launch_batch_d2q9(b->collision, b->storage, b->item_tab, b->items,
                                              src, dst, grid, b->block, b->blocks_per_sm > 0, s);
        if (rc) return rc;
    }
    return LBM_OK;
}

void drop_graph(LbmBatch* b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    b->g_steps = 0;
}

}  // namespace

extern "C" {

int lbm_batch_create(const LbmDesc* lattices, int count, LbmBatch** out) {
    if (lattices == nullptr || out == nullptr) return LBM_E_NULL;
    if (count < 1 || count > 65536) return LBM_E_ARG;
    *out = nullptr;
    const LbmDesc& d0 = lattices[0];
    std::vector<lbm::BatchLattice> host(count);
    auto* b = new LbmBatch();
    b->count = count;
    b->collision = d0.collision;
    b->storage = d0.storage;
    const int V = vec_elems(d0.storage);
    long long base = 0, items = 0;
    for (int l = 0; l < count; ++l) {
        const LbmDesc& d = lattices[l];
        int rc = lbm_validate(&d);
        if (!rc && (d.lattice != LBM_D2Q9 || d.collision != d0.collision ||
                    d.storage != d0.storage || d.collision == LBM_STREAM_ONLY))
            rc = LBM_E_ARG;
        if (!rc && (d.solid_bits || d.force_field || d.mx_force || d.fx != 0.0f || d.fy != 0.0f ||
                    d.inlet_u || d.outlet))
            rc = LBM_E_ARG;  // batches are plain boxes
        if (!rc && d.nx % V != 0) rc = LBM_E_SHAPE;
        if (rc) {
            delete b;
            return rc;
        }
        lbm::BatchLattice& t = host[l];
        t.base = base;
        t.nx = d.nx;
        t.ny = d.ny;
        t.periodic_mask = d.periodic_mask;
        t.segs = d.nx / V;  // vectors per row; a work item is 32 consecutive vectors
        t.item0 = int(items);
        t.ulid = d.ulid;
        t.r0 = d.r0;
        t.r1 = d.r1;
        t.r2 = d.r2;
        t.r3 = d.r3;
        b->bases.push_back(base);
        base += 9LL * d.nx * d.ny;
        b->nodes += (long long)d.nx * d.ny;
        items += ((long long)d.ny * t.segs + 31) / 32;
        if (items >= (1LL << 31)) {
            delete b;
            return LBM_E_SIZE;
        }
    }
    b->elements = base;
    b->items = int(items);
    // one copy of the lattice parameters per work item: a warp's parameters are one load
    // away (no lattice lookup first); 48 bytes per 32 row vectors, read from L2
    std::vector<lbm::BatchLattice> owner(size_t(b->items));
    for (int l = 0; l < count; ++l) {
        const int end = l + 1 < count ? host[l + 1].item0 : b->items;
        for (int k = host[l].item0; k < end; ++k) {
            lbm::BatchLattice& it = owner[size_t(k)];
            it = host[l];
            const long long first = (long long)(k - host[l].item0) * 32;  // first vector
            it.y0 = int(first / host[l].segs);
            it.xv0 = int(first - (long long)it.y0 * host[l].segs);
        }
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&b->item_tab),
                               sizeof(lbm::BatchLattice) * owner.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(b->item_tab, owner.data(), sizeof(lbm::BatchLattice) * owner.size(),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (b->item_tab) cudaFree(b->item_tab);
        delete b;
        return int(e);
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_destroy(LbmBatch* b) {
    if (b == nullptr) return LBM_E_HANDLE;
    drop_graph(b);
    if (b->item_tab) cudaFree(b->item_tab);
    delete b;
    return LBM_OK;
}

int lbm_batch_info(const LbmBatch* b, int64_t* elements, int64_t* nodes, int* items) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (!elements || !nodes || !items) return LBM_E_NULL;
    *elements = b->elements;
    *nodes = b->nodes;
    *items = b->items;
    return LBM_OK;
}

int lbm_batch_offsets(const LbmBatch* b, int64_t* bases) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (!bases) return LBM_E_NULL;
    for (int l = 0; l < b->count; ++l) bases[l] = b->bases[l];
    return LBM_OK;
}

int lbm_batch_set_launch(LbmBatch* b, int block, int blocks_per_sm) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (block != 64 && block != 128 && block != 256) return LBM_E_ARG;
    if (blocks_per_sm < 0 || blocks_per_sm > 64) return LBM_E_ARG;
    if (block != b->block || blocks_per_sm != b->blocks_per_sm) drop_graph(b);
    b->block = block;
    b->blocks_per_sm = blocks_per_sm;
    return LBM_OK;
}

int lbm_batch_get_launch(const LbmBatch* b, int* block, int* blocks_per_sm) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (!block || !blocks_per_sm) return LBM_E_NULL;
    *block = b->block;
    *blocks_per_sm = b->blocks_per_sm;
    return LBM_OK;
}

int lbm_batch_step(LbmBatch* b, void* a, void* bb, int nsteps, uint64_t stream) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (a == nullptr || bb == nullptr) return LBM_E_NULL;
    if (a == bb) return LBM_E_ALIAS;
    if ((reinterpret_cast<uintptr_t>(a) & 15u) || (reinterpret_cast<uintptr_t>(bb) & 15u))
        return LBM_E_ALIGN;
    if (nsteps < 0) return LBM_E_STEPS;
    return launch_steps(b, a, bb, nsteps, reinterpret_cast<cudaStream_t>(stream));
}

int lbm_batch_graph_launch(LbmBatch* b, void* a, void* bb, int nsteps, uint64_t stream) {
    if (b == nullptr) return LBM_E_HANDLE;
    if (a == nullptr || bb == nullptr) return LBM_E_NULL;
    if (a == bb) return LBM_E_ALIAS;
    if ((reinterpret_cast<uintptr_t>(a) & 15u) || (reinterpret_cast<uintptr_t>(bb) & 15u))
        return LBM_E_ALIGN;
    if (nsteps < 1) return LBM_E_STEPS;
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int grid = grid_of(*b);
    if (!(b->exec && b->g_a == a && b->g_b == bb && b->g_steps == nsteps &&
          b->g_block == b->block && b->g_grid == grid)) {
        drop_graph(b);
        cudaStream_t cap;
        cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) return int(e);
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        int rc = (e == cudaSuccess) ? launch_steps(b, a, bb, nsteps, cap) : int(e);
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(cap, &g);
        if (!rc && e2 != cudaSuccess) rc = int(e2);
        if (!rc) {
            e = cudaGraphInstantiate(&b->exec, g, 0);
            if (e != cudaSuccess) rc = int(e);
        }
        if (g) cudaGraphDestroy(g);
        cudaStreamDestroy(cap);
        if (rc) {
            b->exec = nullptr;
            return rc;
        }
        b->g_a = a;
        b->g_b = bb;
        b->g_steps = nsteps;
        b->g_block = b->block;
        b->g_grid = grid;
    }
    return int(cudaGraphLaunch(b->exec, s));
}

}  // extern "C"
