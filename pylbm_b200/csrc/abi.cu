// C ABI entry points: argument validation and dispatch to the kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/pylbm_b200.h"
#include "dispatch.cuh"
#include "lattice.cuh"

using namespace lbm;

namespace lbm {

namespace {
// [lattice][16-bit storage]: row-segment width, ring depth, consumer warps
StagedTune g_tune[2][2] = {{{512, 4, 4}, {1024, 4, 4}}, {{256, 4, 4}, {512, 4, 4}}};
}  // namespace

StagedTune staged_tune(int lattice, int elem_bytes) {
    return g_tune[lattice == LBM_D3Q19 ? 1 : 0][elem_bytes == 2 ? 1 : 0];
}

}  // namespace lbm

namespace {

bool finite(float v) { return std::isfinite(v); }

bool rate_ok(float r) { return std::isfinite(r) && r > 0.0f && r < 2.0f; }

int q_of(int lattice) { return lattice == LBM_D2Q9 ? 9 : 19; }

int elem_size(int storage) {
    return (storage == LBM_STORE_F16 || storage == LBM_STORE_BF16) ? 2 : 4;
}

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

cudaStream_t as_stream(uint64_t s) { return reinterpret_cast<cudaStream_t>(s); }

int launch_one(const LbmDesc& d, const void* src, void* dst, int pattern, cudaStream_t s) {
    if (d.flags & LBM_FLAG_GENERIC)
        return d.lattice == LBM_D2Q9 ? launch_generic_d2q9(d, src, dst, pattern, s)
                                     : launch_generic_d3q19(d, src, dst, pattern, s);
    const int fast = d.lattice == LBM_D2Q9 ? launch_fast_d2q9(d, src, dst, pattern, s)
                                           : launch_fast_d3q19(d, src, dst, pattern, s);
    if (fast != 1) return fast;
    return d.lattice == LBM_D2Q9 ? launch_generic_d2q9(d, src, dst, pattern, s)
                                 : launch_generic_d3q19(d, src, dst, pattern, s);
}

int check_buffer(const LbmDesc& d, const void* p) {
    if (p == nullptr) return LBM_E_NULL;
    if (!aligned(p, uintptr_t(elem_size(d.storage)))) return LBM_E_ALIGN;
    return LBM_OK;
}

int check_pattern(const LbmDesc& d, const void* src, const void* dst, int pattern) {
    if (pattern < LBM_PATTERN_AB || pattern > LBM_PATTERN_AA_EVEN) return LBM_E_PATTERN;
    int rc = check_buffer(d, src);
    if (rc) return rc;
    rc = check_buffer(d, dst);
    if (rc) return rc;
    if (pattern == LBM_PATTERN_AB && src == dst) return LBM_E_ALIAS;
    if (pattern != LBM_PATTERN_AB && src != dst) return LBM_E_ALIAS;
    // solids and the momentum-exchange sum need the two-buffer pull: an AA push cannot keep
    // each memory slot owned by one node once a link is blocked on one side only
    if (pattern != LBM_PATTERN_AB && (d.solid_bits != nullptr || d.mx_force != nullptr))
        return LBM_E_ARG;
    if (pattern != LBM_PATTERN_AB && (d.inlet_u != nullptr || d.outlet)) return LBM_E_INOUT;
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

int lbm_set_staged_config(int lattice, int elem_bytes, int width, int stages, int warps) {
    if (lattice != LBM_D2Q9 && lattice != LBM_D3Q19) return LBM_E_LATTICE;
    if (elem_bytes != 2 && elem_bytes != 4) return LBM_E_STORAGE;
    if (width < 8 || width > 4096 || (width % 8) != 0) return LBM_E_ARG;
    if (stages < 2 || stages > 8 || warps < 1 || warps > 8) return LBM_E_ARG;
    const int q = q_of(lattice);
    const long long smem = 128 + (long long)stages * q * (width + 2 * (16 / elem_bytes)) * elem_bytes;
    if (smem > 227 * 1024) return LBM_E_SIZE;
    g_tune[lattice == LBM_D3Q19 ? 1 : 0][elem_bytes == 2 ? 1 : 0] = {width, stages, warps};
    return LBM_OK;
}

int lbm_get_staged_config(int lattice, int elem_bytes, int* width, int* stages, int* warps) {
    if (lattice != LBM_D2Q9 && lattice != LBM_D3Q19) return LBM_E_LATTICE;
    if (elem_bytes != 2 && elem_bytes != 4) return LBM_E_STORAGE;
    if (!width || !stages || !warps) return LBM_E_NULL;
    const StagedTune t = staged_tune(lattice, elem_bytes);
    *width = t.width;
    *stages = t.stages;
    *warps = t.warps;
    return LBM_OK;
}

int lbm_device_error(int clear) {
    unsigned int bits = 0;
    const int rc = read_device_error(clear, &bits);
    if (rc) return rc;
    return bits ? LBM_E_TIMEOUT : LBM_OK;
}

int lbm_selftest_wait_timeout(const LbmDesc* d, void* buf, uint64_t timeout_ns,
                              uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if (d->lattice != LBM_D3Q19) return LBM_E_LATTICE;
    if ((rc = check_buffer(*d, buf))) return rc;
    if (timeout_ns == 0 || timeout_ns > 10000000000ull) return LBM_E_ARG;
    return launch_staged_timeout_probe(*d, buf, timeout_ns, as_stream(stream));
}

const char* lbm_error_string(int code) {
    switch (code) {
        case LBM_OK: return "success";
        case LBM_E_NULL: return "a required pointer is NULL";
        case LBM_E_LATTICE: return "unknown lattice";
        case LBM_E_COLLISION: return "unknown collision operator";
        case LBM_E_STORAGE: return "unknown storage format";
        case LBM_E_PATTERN: return "unknown streaming pattern";
        case LBM_E_SHAPE: return "invalid lattice shape";
        case LBM_E_INDEX: return "q * N does not fit in int32 indexing";
        case LBM_E_RATE: return "relaxation rate outside (0, 2) or non-finite scalar";
        case LBM_E_LID: return "a moving lid needs a wall on the last axis";
        case LBM_E_ALIGN: return "misaligned device pointer";
        case LBM_E_ALIAS: return "buffer aliasing does not match the pattern";
        case LBM_E_STEPS: return "invalid step count (AA pattern advances in pairs)";
        case LBM_E_TIMEOUT: return "a bounded device-side wait timed out";
        case LBM_E_HANDLE: return "unknown or destroyed handle";
        case LBM_E_ARG: return "invalid argument";
        case LBM_E_SIZE: return "problem exceeds a fixed capacity";
        case LBM_E_INOUT:
            return "inlet and outlet boundaries need D2Q9, walls on the x axis and the AB pattern";
    }
    if (code > 0) return cudaGetErrorString(static_cast<cudaError_t>(code));
    return "unknown error";
}

int lbm_lattice_info(int lattice, int* q, int* dim, int* c, double* w, int* opp) {
    if (lattice != LBM_D2Q9 && lattice != LBM_D3Q19) return LBM_E_LATTICE;
    if (!q || !dim || !c || !w || !opp) return LBM_E_NULL;
    auto fill = [&](auto lat) {
        using L = decltype(lat);
        *q = L::Q;
        *dim = L::D;
        for (int i = 0; i < L::Q; ++i) {
            c[3 * i] = L::cx(i);
            c[3 * i + 1] = L::cy(i);
            c[3 * i + 2] = L::cz(i);
            w[i] = L::wd(i);
            opp[i] = L::opp(i);
        }
    };
    if (lattice == LBM_D2Q9) fill(D2Q9{});
    else fill(D3Q19{});
    return LBM_OK;
}

int lbm_validate(const LbmDesc* d) {
    if (d == nullptr) return LBM_E_NULL;
    if (d->lattice != LBM_D2Q9 && d->lattice != LBM_D3Q19) return LBM_E_LATTICE;
    if (d->collision < LBM_BGK || d->collision > LBM_STREAM_ONLY) return LBM_E_COLLISION;
    if (d->storage < LBM_STORE_F32 || d->storage > LBM_STORE_F32_SHIFTED) return LBM_E_STORAGE;
    const int dim = d->lattice == LBM_D2Q9 ? 2 : 3;
    if (d->nx < 1 || d->ny < 1 || d->nz < 1) return LBM_E_SHAPE;
    if (dim == 2 && d->nz != 1) return LBM_E_SHAPE;
    if (d->ny > 65535 || d->nz > 65535) return LBM_E_SHAPE;  // grid.y / grid.z limits
    const long long N = (long long)d->nx * d->ny * d->nz;
    if ((long long)q_of(d->lattice) * N >= (1LL << 31)) return LBM_E_INDEX;
    if (d->collision != LBM_STREAM_ONLY && !rate_ok(d->r0)) return LBM_E_RATE;
    if (d->collision == LBM_TRT && !rate_ok(d->r1)) return LBM_E_RATE;
    if (d->collision == LBM_MRT && (!rate_ok(d->r1) || !rate_ok(d->r2) || !rate_ok(d->r3)))
        return LBM_E_RATE;
    if (!finite(d->ulid) || !finite(d->fx) || !finite(d->fy) || !finite(d->fz))
        return LBM_E_RATE;
    if (d->ulid != 0.0f && ((d->periodic_mask >> (dim - 1)) & 1)) return LBM_E_LID;
    if (d->solid_bits && !aligned(d->solid_bits, 4)) return LBM_E_ALIGN;
    if (d->force_field && !aligned(d->force_field, 4)) return LBM_E_ALIGN;
    if (d->mx_force) {
        if (!aligned(d->mx_force, 8)) return LBM_E_ALIGN;
        if (!d->solid_bits) return LBM_E_ARG;
    }
    if (d->mx_stride < 0) return LBM_E_ARG;
    if (d->outlet != 0 && d->outlet != 1) return LBM_E_ARG;
    if (d->inlet_u || d->outlet) {
        if (d->lattice != LBM_D2Q9 || (d->periodic_mask & 1) || d->nx < 3) return LBM_E_INOUT;
        if (d->inlet_u && !aligned(d->inlet_u, 4)) return LBM_E_ALIGN;
    }
    return LBM_OK;
}

int lbm_launch(const LbmDesc* d, const void* src, void* dst, int pattern, uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if (dst == nullptr && pattern != LBM_PATTERN_AB) dst = const_cast<void*>(src);
    rc = check_pattern(*d, src, dst, pattern);
    if (rc) return rc;
    return launch_one(*d, src, dst, pattern, as_stream(stream));
}

int lbm_advance(const LbmDesc* d, void* a, void* b, int aa, int nsteps, uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if (nsteps < 0) return LBM_E_STEPS;
    if (aa && (nsteps & 1)) return LBM_E_STEPS;
    rc = aa ? check_pattern(*d, a, a, LBM_PATTERN_AA_ODD) : check_pattern(*d, a, b, LBM_PATTERN_AB);
    if (rc) return rc;
    const cudaStream_t s = as_stream(stream);
    LbmDesc step = *d;
    for (int k = 0; k < nsteps; ++k) {
        if (aa) {
            rc = launch_one(step, a, a, (k & 1) ? LBM_PATTERN_AA_EVEN : LBM_PATTERN_AA_ODD, s);
        } else {
            rc = (k & 1) ? launch_one(step, b, a, LBM_PATTERN_AB, s)
                         : launch_one(step, a, b, LBM_PATTERN_AB, s);
        }
        if (rc) return rc;
        if (step.mx_force) step.mx_force += step.mx_stride;
    }
    return LBM_OK;
}

int lbm_moments_f64(const LbmDesc* d, const void* f, int layout, double* out,
                    uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if ((rc = check_buffer(*d, f))) return rc;
    if (out == nullptr) return LBM_E_NULL;
    if (!aligned(out, 8)) return LBM_E_ALIGN;
    if (layout != LBM_LAYOUT_NATURAL && layout != LBM_LAYOUT_AA_SWAPPED) return LBM_E_ARG;
    return launch_moments(*d, f, layout, out, as_stream(stream));
}

int lbm_macroscopic(const LbmDesc* d, const void* f, int layout, float* rho, float* u,
                    uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if ((rc = check_buffer(*d, f))) return rc;
    if (rho == nullptr || u == nullptr) return LBM_E_NULL;
    if (!aligned(rho, 4) || !aligned(u, 4)) return LBM_E_ALIGN;
    if (layout != LBM_LAYOUT_NATURAL && layout != LBM_LAYOUT_AA_SWAPPED) return LBM_E_ARG;
    return launch_macroscopic(*d, f, layout, rho, u, as_stream(stream));
}

int lbm_encode_f64(const LbmDesc* d, const double* f64, void* buf, int layout,
                   uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if ((rc = check_buffer(*d, buf))) return rc;
    if (f64 == nullptr) return LBM_E_NULL;
    if (!aligned(f64, 8)) return LBM_E_ALIGN;
    if (layout != LBM_LAYOUT_NATURAL && layout != LBM_LAYOUT_AA_SWAPPED) return LBM_E_ARG;
    return launch_encode(*d, f64, buf, layout, as_stream(stream));
}

int lbm_decode_f64(const LbmDesc* d, const void* buf, int layout, double* f64,
                   uint64_t stream) {
    int rc = lbm_validate(d);
    if (rc) return rc;
    if ((rc = check_buffer(*d, buf))) return rc;
    if (f64 == nullptr) return LBM_E_NULL;
    if (!aligned(f64, 8)) return LBM_E_ALIGN;
    if (layout != LBM_LAYOUT_NATURAL && layout != LBM_LAYOUT_AA_SWAPPED) return LBM_E_ARG;
    return launch_decode(*d, buf, layout, f64, as_stream(stream));
}

}  // extern "C"
