// B200 kernels of the inundation shallow-water step: float64 volume, the
// two-sum probe and the Manning power, with their C ABI. The stage kernels
// are in swe_stage.cu, the dilation, clock, prologue and sources in
// swe_control.cu.
//
// Reference: inundation/vulkan/shaders/resident.py (GLSL) driven by
// inundation/vulkan/gpu_resident_batch.py; the per-function comments give
// the lines each kernel replaces.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "swe_common.cuh"

namespace swe {

// ---------------------------------------------------------------------------
// Float64 volume, fixed order: per-CTA partials, then one CTA over them.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads)
    volume_partial_kernel(const float *h, const float *h_lo, const float *area, uint32_t n, uint32_t per_cta, double *partials) {
    __shared__ double acc[kThreads];
    const uint32_t lo = blockIdx.x * per_cta;
    const uint32_t hi = min(n, lo + per_cta);
    double sum = 0.0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += kThreads)
        sum += (static_cast<double>(h[i]) + static_cast<double>(h_lo ? h_lo[i] : 0.0f)) * static_cast<double>(area[i]);
    acc[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) acc[threadIdx.x] += acc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = acc[0];
}

__global__ void __launch_bounds__(kThreads) volume_final_kernel(const double *partials, uint32_t count, double *out) {
    __shared__ double acc[kThreads];
    double sum = 0.0;
    for (uint32_t i = threadIdx.x; i < count; i += kThreads) sum += partials[i];
    acc[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) acc[threadIdx.x] += acc[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = acc[0];
}

__global__ void eft_probe_kernel(float *v) {
    float se, ee;
    two_sum(v[0], v[1], se, ee);
    v[2] = ee;
}

__global__ void inv_pow43_kernel(const float *x, float *out, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = inv_pow43(x[i]);
}

// The ghost state and mass flux of open edges from given cells: the device
// half of the reference's ghost probe (tests/unit/test_gpu_open_ghost.py:45-71).
__global__ void open_ghost_kernel(const float *cases, const uint32_t *cond, float *results, uint32_t n, Phys p) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const float *c = cases + 6ull * k;
        const uint32_t kind = cond[2ull * k];
        const float value = __uint_as_float(cond[2ull * k + 1]);
        float hG, huG, hvG;
        ghost_state(p, kind, value, c[0], c[1], c[2], c[3], c[4], hG, huG, hvG);
        float *r = results + 4ull * k;
        r[0] = hG;
        r[1] = huG;
        r[2] = hvG;
        r[3] = boundary_mass_flux(kind, value, c[5]);
    }
}

// One bounded wait for instance 0's published dt pair (the seats' wait in the
// persistent kernel): the dt bits, or 0 and error bit 4 after the wait limit.
__global__ void dt_wait_probe_kernel(swe_state_t s, uint32_t epoch, uint32_t *out) {
    const uint64_t *pair = dt_pair(s, 0u);
    out[0] = published_dt(s, pair, epoch, ld_relaxed_u64(pair));
}

}  // namespace swe

using namespace swe;

extern "C" {

uint32_t swe_volume_partials(uint32_t n_cells) {
    const uint32_t p = (n_cells + 4095u) / 4096u;
    return p < 1u ? 1u : (p > 1024u ? 1024u : p);
}

int swe_volume_fp64(const float *h, const float *h_lo, const float *area, uint32_t n_cells, double *partials, double *out,
                    swe_stream_t stream) {
    if (!h || !area || !partials || !out || n_cells == 0u) return SWE_ERR_ARGUMENT;
    const uint32_t parts = swe_volume_partials(n_cells);
    const uint32_t per = (n_cells + parts - 1) / parts;
    volume_partial_kernel<<<parts, kThreads, 0, stream>>>(h, h_lo, area, n_cells, per, partials);
    int rc = check_launch();
    if (rc) return rc;
    volume_final_kernel<<<1, kThreads, 0, stream>>>(partials, parts, out);
    return check_launch();
}

int swe_dt_wait_probe(const swe_state_t *state, uint32_t epoch, uint32_t *out, swe_stream_t stream) {
    if (!state || !state->dt_buf || !state->ctrl || !out || (reinterpret_cast<uintptr_t>(state->dt_buf) & 15u))
        return SWE_ERR_ARGUMENT;
    dt_wait_probe_kernel<<<1, 1, 0, stream>>>(*state, epoch, out);
    return check_launch();
}

int swe_eft_probe(float *v, swe_stream_t stream) {
    if (!v) return SWE_ERR_ARGUMENT;
    eft_probe_kernel<<<1, 1, 0, stream>>>(v);
    return check_launch();
}

int swe_inv_pow43(const float *x, float *out, uint32_t n, swe_stream_t stream) {
    if (!x || !out || n == 0u) return SWE_ERR_ARGUMENT;
    inv_pow43_kernel<<<min((n + 255u) / 256u, 4096u), 256, 0, stream>>>(x, out, n);
    return check_launch();
}

int swe_open_ghost_probe(const float *cases, const uint32_t *cond, float *results, uint32_t n, float g,
                         float dry_tol, swe_stream_t stream) {
    if (!cases || !cond || !results || n == 0u) return SWE_ERR_ARGUMENT;
    Phys p;
    p.g = g;
    p.dry_tol = dry_tol;
    open_ghost_kernel<<<min((n + 255u) / 256u, 4096u), 256, 0, stream>>>(cases, cond, results, n, p);
    return check_launch();
}

const char *swe_status_string(int status) {
    switch (status) {
        case SWE_OK: return "ok";
        case SWE_ERR_ARGUMENT: return "invalid argument";
        case SWE_ERR_CUDA: return "CUDA launch or runtime error";
        case SWE_ERR_TOO_LARGE:
            return "size beyond a fixed limit (an edge tile larger than shared memory or than a work item's fields, "
                   "or more cells than the allocation-free volume's static scratch holds)";
        case SWE_ERR_MATH: return "device arithmetic lost the two-sum error term";
        default: return "unknown status";
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free float64 volume.
//
// For callers that must not allocate device memory during a run: a host that
// runs under a fixed device-memory budget checked at start-up, an embedding
// application that owns the CUDA allocator, or code called from a context
// where cudaMalloc is not allowed. The per-CTA partial sums that
// swe_volume_fp64 takes from its caller live here in a static device array
// instead; every GPU that loads this library holds it (8 KiB) until exit.
// ---------------------------------------------------------------------------
namespace swe {

constexpr uint32_t kNoAllocPartials = 1024;
constexpr uint32_t kNoAllocCellsPerPartial = 4096;
constexpr uint32_t kNoAllocMaxCells = kNoAllocPartials * kNoAllocCellsPerPartial;
constexpr int kNoAllocDevices = 64;

static __device__ __align__(256) double g_volume_scratch[kNoAllocPartials];

// Device address of g_volume_scratch per device ordinal. In host code the
// array's name is only a host-side stand-in, never a device address.
static std::atomic<double *> g_volume_scratch_addr[kNoAllocDevices];

}  // namespace swe

extern "C" int swe_volume_fp64_noalloc(const float *h, const float *h_lo, const float *area, uint32_t n_cells,
                                       double *out, swe_stream_t stream) {
    if (!h || !area || !out || n_cells == 0u) return SWE_ERR_ARGUMENT;
    if (n_cells > kNoAllocMaxCells) return SWE_ERR_TOO_LARGE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return SWE_ERR_CUDA;
    if (dev < 0 || dev >= kNoAllocDevices) return SWE_ERR_ARGUMENT;
    double *scratch = g_volume_scratch_addr[dev].load(std::memory_order_acquire);
    if (scratch == nullptr) {
        // First call on this device (the device must be current): look up the
        // array's device address once and keep it for the life of the process
        // (a cudaDeviceReset may load the module elsewhere: see the header).
        void *addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_volume_scratch) != cudaSuccess || addr == nullptr) return SWE_ERR_CUDA;
        scratch = static_cast<double *>(addr);
        g_volume_scratch_addr[dev].store(scratch, std::memory_order_release);
    }
    // Same partition as swe_volume_fp64 (one partial per 4096 cells below the
    // limit), so both entry points sum in the same order. Every partial the
    // final pass reads is rewritten first, so the array needs no clearing.
    const uint32_t parts = swe_volume_partials(n_cells);
    const uint32_t per = (n_cells + parts - 1) / parts;
    volume_partial_kernel<<<parts, kThreads, 0, stream>>>(h, h_lo, area, n_cells, per, scratch);
    int rc = check_launch();
    if (rc) return rc;
    volume_final_kernel<<<1, kThreads, 0, stream>>>(scratch, parts, out);
    return check_launch();
}
