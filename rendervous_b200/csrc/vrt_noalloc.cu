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
//     float each: 1 MiB) after a 512-byte block for the kernel counters.  Every
//     GPU that loads the library keeps this memory until the process exits.
//   - Every call shares the array and overwrites it; the counters are cleared
//     at the start of each call.  Calls whose kernels overlap on the GPU (on
//     different streams, or different host threads) race on it.
//   - The device address of the array is looked up once per device, on the
//     first call made with that device current; make that first call before
//     any stream capture.
#include <cstdint>
#include <cstdio>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_internal.h"

namespace vrt {
namespace {

constexpr int kMaxBricks = 64 * 64 * 64;
constexpr size_t kCounterBytes = 512;
constexpr size_t kScratchBytes = kCounterBytes + sizeof(float) * (size_t)kMaxBricks;
constexpr int kMaxDevices = 64;

static_assert(sizeof(DScratch) <= kCounterBytes, "counter block must fit its slot");

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;
unsigned char* g_base[kMaxDevices] = {};

// Device address of g_scratch for the current device (host code cannot use the
// symbol itself: on the host it names a stand-in, not device memory).
int scratch_base(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return VRT_E_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_base[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "[vrt] cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return VRT_E_CUDA;
        }
        g_base[device] = static_cast<unsigned char*>(p);
    }
    *out = g_base[device];
    return VRT_OK;
}

}  // namespace
}  // namespace vrt

extern "C" int vrt_transmittance_fw_noalloc(const vrt_medium* m, int32_t mode, int32_t brick, const float* rays,
                                            int64_t n, uint64_t seed, float* T, void* stream) {
    using namespace vrt;
    if (!m) return VRT_E_NULL_POINTER;
    if (mode < 0 || mode > 3 || brick < 0) return VRT_E_INVALID_ARGUMENT;
    int device = -1;
    if (cudaGetDevice(&device) != cudaSuccess) return VRT_E_CUDA;
    unsigned char* base = nullptr;
    int st = scratch_base(device, &base);
    if (st) return st;

    vrt_medium mm = *m;
    cudaStream_t s = (cudaStream_t)stream;
    if (brick > 0 && mode <= 1) {
        int32_t dims[3];
        if ((st = vrt_majorant_build(&m->sigma, brick, nullptr, dims, stream))) return st;
        if ((int64_t)dims[0] * dims[1] * dims[2] > kMaxBricks) {
            std::fprintf(stderr,
                         "[vrt] vrt_transmittance_fw_noalloc: %d x %d x %d majorant bricks exceed the fixed "
                         "scratch of %d bricks; use a larger brick or vrt_transmittance_fw\n",
                         dims[0], dims[1], dims[2], kMaxBricks);
            return VRT_E_BAD_SHAPE;
        }
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
    vrt_context ctx;
    ctx.device = device;
    ctx.num_sms = 0;  // unused by the transmittance launch
    ctx.scratch = reinterpret_cast<DScratch*>(base);
    return vrt_transmittance_fw(&ctx, &mm, mode, rays, n, seed, T, stream);
}
