// vrt_noalloc.cu -- transmittance on rays without any device allocation.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or a pre-sized arena, plugins that are not allowed to
// grow the process's device footprint, or hosts that create no CUDA context of
// their own beyond the one they were handed.  For them this file provides one
// entry point, vrt_transmittance_fw_noalloc, that needs no vrt_context and no
// caller-provided scratch: the majorant grid it builds and the counters its
// kernel updates live in a fixed array compiled into libvrt.so.
//
//   - The array holds at most kMaxBricks majorant bricks (64^3 = 262144, one
//     float each: 1 MiB) after a 1024-byte block for the kernel counters.  Every
//     GPU that loads the library keeps this memory until the process exits.
//   - Every call shares the array and overwrites it; the counters are cleared
//     at the start of each call.  Calls whose kernels overlap on the GPU (on
//     different streams, or different host threads) race on it.
//   - The device address of the array is looked up once per CUDA context, on
//     the first call made with that context current, and cached under the
//     context's unique id (a context created after cudaDeviceReset, or another
//     context on the same device, gets its own lookup).  Make that first call
//     before any stream capture.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_internal.h"

namespace vrt {
namespace {

constexpr int kMaxBricks = 64 * 64 * 64;
constexpr size_t kCounterBytes = 1024;
constexpr size_t kScratchBytes = kCounterBytes + sizeof(float) * (size_t)kMaxBricks;
constexpr int kCacheSlots = 64;

static_assert(sizeof(DScratch) <= kCounterBytes, "counter block must fit its slot");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Driver calls reached through the runtime (no link against libcuda).
typedef CUresult (*PFN_ctx_current)(CUcontext*);
typedef CUresult (*PFN_ctx_id)(CUcontext, unsigned long long*);

std::mutex g_mutex;
bool g_resolved = false;
PFN_ctx_current g_ctx_current = nullptr;
PFN_ctx_id g_ctx_id = nullptr;
struct Slot {
    unsigned long long ctx_id;
    unsigned char* base;
};
Slot g_slots[kCacheSlots] = {};
int g_nslots = 0;

// Unique id of the calling thread's current context; false if the driver
// entry points are unavailable or no context is current.
bool current_context_id(unsigned long long* id) {
    if (!g_resolved) {
        g_resolved = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_current = reinterpret_cast<PFN_ctx_current>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_id = reinterpret_cast<PFN_ctx_id>(f);
        cudaGetLastError();
    }
    if (!g_ctx_current || !g_ctx_id) return false;
    CUcontext c = nullptr;
    if (g_ctx_current(&c) != CUDA_SUCCESS || !c) return false;
    return g_ctx_id(c, id) == CUDA_SUCCESS;
}

// Device address of g_scratch in the current context (host code cannot use
// the symbol itself: on the host it names a stand-in, not device memory).
int scratch_base(unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_mutex);
    unsigned long long id = 0;
    const bool have_id = current_context_id(&id);
    if (have_id)
        for (int i = 0; i < g_nslots; ++i)
            if (g_slots[i].ctx_id == id) {
                *out = g_slots[i].base;
                return VRT_OK;
            }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[vrt] cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return VRT_E_CUDA;
    }
    // the id is only re-read once it was found; without one the address is
    // looked up on every call (still no allocation)
    if (have_id && g_nslots < kCacheSlots) g_slots[g_nslots++] = {id, static_cast<unsigned char*>(p)};
    *out = static_cast<unsigned char*>(p);
    return VRT_OK;
}

}  // namespace
}  // namespace vrt

extern "C" int vrt_transmittance_fw_noalloc(const vrt_medium* m, int32_t mode, int32_t brick, const float* rays,
                                            int64_t n, uint64_t seed, float* T, int64_t* status_out, void* stream) {
    using namespace vrt;
    if (status_out) *status_out = 0;
    // every argument check comes before the first launch, so a call that is
    // refused leaves the shared array (and any call still using it) untouched
    if (!m) return VRT_E_NULL_POINTER;
    if (mode < 0 || mode > 3 || brick < 0) return VRT_E_INVALID_ARGUMENT;
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!rays || !T) return VRT_E_NULL_POINTER;
    if (((uintptr_t)rays & 7u) != 0) return VRT_E_INVALID_ARGUMENT;
    int32_t dims[3] = {0, 0, 0};
    const bool own_majorant = brick > 0 && mode <= 1;
    int st;
    if (own_majorant) {
        if ((st = vrt_majorant_build(&m->sigma, brick, nullptr, dims, stream))) return st;  // sizes only
        if ((int64_t)dims[0] * dims[1] * dims[2] > kMaxBricks) {
            std::fprintf(stderr,
                         "[vrt] vrt_transmittance_fw_noalloc: %d x %d x %d majorant bricks exceed the fixed "
                         "scratch of %d bricks; use a larger brick or vrt_transmittance_fw\n",
                         dims[0], dims[1], dims[2], kMaxBricks);
            return VRT_E_BAD_SHAPE;
        }
    }
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess) return VRT_E_CUDA;
    unsigned char* base = nullptr;
    if ((st = scratch_base(&base))) return st;

    vrt_medium mm = *m;
    cudaStream_t s = (cudaStream_t)stream;
    if (own_majorant) {
        float* maj = reinterpret_cast<float*>(base + kCounterBytes);
        if ((st = vrt_majorant_build(&m->sigma, brick, maj, dims, stream))) return st;
        mm.majorant_mode = 1;
        mm.maj_grid = maj;
        const int32_t shape[3] = {m->sigma.shape[2], m->sigma.shape[1], m->sigma.shape[0]};  // W, H, D
        for (int i = 0; i < 3; ++i) {
            mm.maj_dims[i] = dims[i];
            mm.maj_scale[i] = m->inv_bsize[i] * (float)(shape[i] - 1) / (float)brick;
        }
    }
    // counters and error word start at zero for this call
    cudaError_t e = cudaMemsetAsync(base, 0, sizeof(DScratch), s);
    if (e != cudaSuccess) return launch_status(e);
    vrt_context ctx{};
    ctx.device = device;
    ctx.scratch = reinterpret_cast<DScratch*>(base);
    if ((st = vrt_transmittance_fw(&ctx, &mm, mode, rays, n, seed, T, stream))) return st;
    if (!status_out) return VRT_OK;
    // the caller asked for the device error word: wait for this call's kernels
    // and copy it out of the shared array (into pageable host memory)
    uint32_t bits = 0;
    DScratch* d = reinterpret_cast<DScratch*>(base);
    if ((e = cudaMemcpyAsync(&bits, &d->status, sizeof(bits), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return launch_status(e);
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return launch_status(e);
    *status_out = (int64_t)bits;
    for (int code = 1; code < 8; ++code)
        if (bits & (1u << code)) return code;
    return VRT_OK;
}
