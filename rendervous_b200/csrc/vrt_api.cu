// vrt_api.cu -- the extern "C" entry points of libvrt.so (declared in include/vrt.h).
//
// Each entry point validates its arguments on the host (null pointers, shapes,
// strides, modes, alignment) before any launch, converts the C structs into the
// kernel-parameter forms of vrt_params.h and launches on the caller's stream.
// There is no CPU fallback: every computation is a CUDA kernel.
#include <atomic>
#include <mutex>
#include <vector>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"

namespace vrt {

int launch_status(cudaError_t e) {
    if (e == cudaSuccess) return VRT_OK;
    std::fprintf(stderr, "[vrt] CUDA error: %s\n", cudaGetErrorString(e));
    return VRT_E_CUDA;
}

static std::atomic<long long> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

// Per-kernel launch counts and (optional) event timing of the wavefront kernels.
namespace {
struct KernelTiming {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Pending {
        int kid;
        cudaEvent_t e0, e1;
    };
    std::vector<Pending> pending;
    long long launches[VRT_K_COUNT] = {};
};
KernelTiming& timing() {
    static KernelTiming t;
    return t;
}
cudaEvent_t take_event(KernelTiming& t) {
    if (!t.pool.empty()) {
        cudaEvent_t e = t.pool.back();
        t.pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}
}  // namespace

KernelScope::KernelScope(int k, cudaStream_t s) : kid(k), stream(s), e0(nullptr), e1(nullptr) {
    KernelTiming& t = timing();
    std::lock_guard<std::mutex> lock(t.mu);
    ++t.launches[kid];
    if (!t.on) return;
    e0 = take_event(t);
    e1 = take_event(t);
    if (e0) cudaEventRecord(e0, stream);
}

KernelScope::~KernelScope() {
    if (!e0 || !e1) return;
    KernelTiming& t = timing();
    std::lock_guard<std::mutex> lock(t.mu);
    cudaEventRecord(e1, stream);
    t.pending.push_back({kid, e0, e1});
}

// The wavefront serves the NEE forward, capped or not (an uncapped path walks
// at most kUncappedPass vertices per round and resumes in the next).
static bool use_wave(const DMedium& M, int integrator) {
    return integrator == VRT_PI_NEE && M.max_bounces <= 4096;
}
// The NEE_DS adjoint wavefront reuses the primal's shadow transmittances in the
// replay, which retraces the primal only with the default replay majorant;
// uncapped paths longer than kUncappedPass vertices finish on the state machine.
static bool use_wave_bw(const DMedium& M, int bw_mode) {
    return bw_mode == VRT_BW_NEE_DS && M.max_bounces <= 4096 && !M.ds_compat;
}
// the DRT, DRTDS and DRTQ adjoints on the wavefront (capped or not): ratio / delta tracking light rays
static bool use_wave_drt(const DMedium& M, int bw_mode) {
    return (bw_mode == VRT_BW_NEE_DRT || bw_mode == VRT_BW_NEE_DRTDS || bw_mode == VRT_BW_NEE_DRTQ) &&
           M.max_bounces <= 4096 && M.tr_mode <= 1;
}
// the SPS adjoint on the wavefront (capped or not): ratio / delta tracking light rays
static bool use_wave_sps(const DMedium& M, int bw_mode) {
    return bw_mode == VRT_BW_NEE_SPS && M.max_bounces <= 4096 && M.tr_mode <= 1;
}

static bool is_collision(int integrator) {
    return integrator == VRT_PI_MC_COLLISION || integrator == VRT_PI_DDA_COLLISION;
}
static int collision_of(int bw_mode) {
    return bw_mode == VRT_BW_MC_COLLISION ? VRT_PI_MC_COLLISION : VRT_PI_DDA_COLLISION;
}

int ensure_wave_buffer(vrt_context* ctx, size_t bytes) {
    if (ctx->wave && ctx->wave_bytes >= bytes) return VRT_OK;
    if (ctx->wave) {
        cudaFree(ctx->wave);
        ctx->wave = nullptr;
        ctx->wave_bytes = 0;
    }
    if (cudaMalloc(&ctx->wave, bytes) != cudaSuccess) {
        cudaGetLastError();
        ctx->wave = nullptr;
        return VRT_E_CUDA;
    }
    ctx->wave_bytes = bytes;
    return VRT_OK;
}

int persistent_blocks(const void* kernel, int block, int num_sms) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

// ---------------------------------------------------------------- kernels --
// Random 32-byte gathers (one L2 sector each, L1 bypassed) over `sectors`
// sectors: four independent address chains per thread keep loads in flight;
// every loaded word feeds the result, so no load can be dropped.
__global__ void __launch_bounds__(256) k_gather_peak(const uint4* __restrict__ buf, unsigned long long sectors,
                                                     int per_thread, uint32_t seed, unsigned int* sink) {
    uint32_t h[4];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int c = 0; c < 4; ++c) h[c] = (t * 4u + (uint32_t)c) * 2654435761u ^ seed;
    uint32_t acc = 0;
    for (int i = 0; i < per_thread; i += 4) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            h[c] = h[c] * 1664525u + 1013904223u;  // LCG (Numerical Recipes constants)
            const unsigned long long s = ((unsigned long long)(h[c] ^ (h[c] >> 15)) * sectors) >> 32;
            const uint4 a = __ldcg(buf + 2 * s), b = __ldcg(buf + 2 * s + 1);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w;  // every loaded byte is used
        }
    }
    if (acc == 0x9e3779b9u) atomicAdd(sink, 1u);
}

// Random float atomic adds (red.global.add, the result unused) over n words:
// four independent address chains per thread; pairs: one vector atomic adds
// two x-neighbours (the scatter form of the adjoints).
__global__ void __launch_bounds__(256) k_atomic_peak(float* __restrict__ buf, unsigned long long n, int per_thread,
                                                     int pairs, uint32_t seed) {
    uint32_t h[4];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int c = 0; c < 4; ++c) h[c] = (t * 4u + (uint32_t)c) * 2654435761u ^ seed;
    const float v = 1.0f / 1048576.0f;
    for (int i = 0; i < per_thread; i += 4) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            h[c] = h[c] * 1664525u + 1013904223u;  // LCG (Numerical Recipes constants)
            if (pairs) {
                const unsigned long long s = ((unsigned long long)(h[c] ^ (h[c] >> 15)) * (n / 2)) >> 32;
                atomicAdd(reinterpret_cast<float2*>(buf) + s, make_float2(v, v));
            } else {
                const unsigned long long s = ((unsigned long long)(h[c] ^ (h[c] >> 15)) * n) >> 32;
                atomicAdd(buf + s, v);
            }
        }
    }
}

__global__ void k_ray_box(const float* __restrict__ rays, int64_t n, float3 bmin, float3 bmax, float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float tMin, tMax;
        ray_box_intersection(ld3(rays + 6 * i), ld3(rays + 6 * i + 3), bmin, bmax, tMin, tMax);
        out[2 * i] = tMin;
        out[2 * i + 1] = tMax;
    }
}

// Grid3D FORWARD for any channel count (include/maps/grid3d.h:6-37)
__global__ void k_grid_fw(DGrid g, float3 bmin, float3 inv_bsize, const float* __restrict__ x, int64_t n,
                          float* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float3 c = ld3(x + 3 * i);
        float3 nc = make_float3((c.x - bmin.x) * inv_bsize.x, (c.y - bmin.y) * inv_bsize.y, (c.z - bmin.z) * inv_bsize.z);
        float* o = out + (int64_t)g.C * i;
        for (int k = 0; k < g.C; ++k) o[k] = 0.0f;
        if (nc.x < 0.0f || nc.y < 0.0f || nc.z < 0.0f || nc.x >= 1.0f || nc.y >= 1.0f || nc.z >= 1.0f) continue;
        const int dx = g.W - 1, dy = g.H - 1, dz = g.D - 1;
        float gx = nc.x * (float)dx, gy = nc.y * (float)dy, gz = nc.z * (float)dz;
        float ax = gx - floorf(gx), ay = gy - floorf(gy), az = gz - floorf(gz);
        int px = min(max((int)gx, 0), dx - 1), py = min(max((int)gy, 0), dy - 1), pz = min(max((int)gz, 0), dz - 1);
        const float* b = g.data + (pz * g.sD + py * g.sH + px * g.sW);
        float bx = 1.0f - ax, by = 1.0f - ay, bz = 1.0f - az;
        const int off[8] = {0, g.sW, g.sH, g.sH + g.sW, g.sD, g.sD + g.sW, g.sD + g.sH, g.sD + g.sH + g.sW};
        const float wt[8] = {bx * by * bz, ax * by * bz, bx * ay * bz, ax * ay * bz,
                             bx * by * az, ax * by * az, bx * ay * az, ax * ay * az};
        for (int k = 0; k < g.C; ++k) {
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < 8; ++j) acc += __ldg(b + off[j] + k) * wt[j];
            o[k] = acc;
        }
    }
}

// Grid3D BACKWARD (include/maps/grid3d.h:39-75)
__global__ void k_grid_bw(DGrid g, float3 bmin, float3 inv_bsize, const float* __restrict__ x,
                          const float* __restrict__ dout, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float3 c = ld3(x + 3 * i);
        float3 nc = make_float3((c.x - bmin.x) * inv_bsize.x, (c.y - bmin.y) * inv_bsize.y, (c.z - bmin.z) * inv_bsize.z);
        grid_scatter(g, nc, dout + (int64_t)g.C * i, g.C);
    }
}

// Majorant grid: brick b bounds nodes [b*B-1, (b+1)*B+1] clamped to the grid.
// One warp per brick; lanes stride over the brick's nodes, then reduce.
__global__ void k_majorant_build(DGrid g, int brick, int Mx, int My, int Mz, float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t total = (int64_t)Mx * My * Mz;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int dim[3] = {g.W - 1, g.H - 1, g.D - 1};
    for (int64_t b = warp; b < total; b += nwarps) {
        int mx = (int)(b % Mx), my = (int)((b / Mx) % My), mz = (int)(b / ((int64_t)Mx * My));
        int lo[3] = {max(mx * brick - 1, 0), max(my * brick - 1, 0), max(mz * brick - 1, 0)};
        int hi[3] = {min((mx + 1) * brick + 1, dim[0]), min((my + 1) * brick + 1, dim[1]), min((mz + 1) * brick + 1, dim[2])};
        int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
        int cnt = nx * ny * nz;
        float m = 0.0f;
        for (int k = lane; k < cnt; k += 32) {
            int xx = lo[0] + k % nx, yy = lo[1] + (k / nx) % ny, zz = lo[2] + k / (nx * ny);
            m = fmaxf(m, __ldg(g.data + zz * g.sD + yy * g.sH + xx * g.sW));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) out[b] = m;
    }
}

static int blocks_for(int64_t n, int per = 256) {
    int64_t b = (n + per - 1) / per;
    if (b < 1) b = 1;
    return (int)(b < 65535 * 8 ? b : 65535 * 8);
}

// ------------------------------------------------------------- validation --
static bool finite3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

static int to_dgrid(const vrt_grid& g, int need_c, DGrid& out) {
    if (!g.data) return VRT_E_NULL_POINTER;
    for (int i = 0; i < 3; ++i)
        if (g.shape[i] < 2) return VRT_E_BAD_SHAPE;
    if (g.shape[3] < 1 || (need_c > 0 && g.shape[3] != need_c)) return VRT_E_BAD_SHAPE;
    if (g.shape[3] > 1 && g.strides[3] != 1) return VRT_E_BAD_SHAPE;
    int64_t max_off = 0;
    for (int i = 0; i < 3; ++i) {
        if (g.strides[i] < 0) return VRT_E_BAD_SHAPE;
        max_off += (int64_t)(g.shape[i] - 1) * g.strides[i];
    }
    max_off += g.shape[3] - 1;
    if (max_off >= (int64_t)INT32_MAX) return VRT_E_BAD_SHAPE;
    out.data = g.data;
    out.grad = g.grad;
    out.D = g.shape[0]; out.H = g.shape[1]; out.W = g.shape[2]; out.C = g.shape[3];
    out.sD = (int)g.strides[0]; out.sH = (int)g.strides[1]; out.sW = (int)g.strides[2];
    return VRT_OK;
}

static float3 mk3(const float* v) { return make_float3(v[0], v[1], v[2]); }

static int to_dmedium(const vrt_medium* m, DMedium& M) {
    if (!m) return VRT_E_NULL_POINTER;
    std::memset(&M, 0, sizeof(M));
    int st = to_dgrid(m->sigma, 1, M.sigma);
    if (st) return st;
    if (m->albedo_is_grid) {
        st = to_dgrid(m->albedo, 0, M.albedo);
        if (st) return st;
        if (M.albedo.C != 1 && M.albedo.C != 3) return VRT_E_BAD_SHAPE;
    }
    const float* vecs[] = {m->bmin, m->bmax, m->inv_bsize, m->box_min, m->box_max, m->albedo_const, m->emission,
                           m->env, m->sun_dir, m->sun_radiance};
    for (const float* v : vecs)
        if (!finite3(v)) return VRT_E_NONFINITE;
    if (!std::isfinite(m->phase_g) || !std::isfinite(m->ds_epsilon) || !std::isfinite(m->global_majorant))
        return VRT_E_NONFINITE;
    if (m->phase_mode < 0 || m->phase_mode > 1) return VRT_E_INVALID_ARGUMENT;
    if (m->transmittance_mode < 0 || m->transmittance_mode > 5) return VRT_E_INVALID_ARGUMENT;
    if (m->max_bounces < 0) return VRT_E_INVALID_ARGUMENT;
    if (m->exitance_mode < 0 || m->exitance_mode > 2) return VRT_E_INVALID_ARGUMENT;
    if (m->env_mode < 0 || m->env_mode > 1 || m->env_sampler < 0 || m->env_sampler > 1) return VRT_E_INVALID_ARGUMENT;
    if (m->env_mode == 1) {
        if (!m->env_image) return VRT_E_NULL_POINTER;
        if (m->env_hw[0] < 1 || m->env_hw[1] < 1 || (int64_t)m->env_hw[0] * m->env_hw[1] * 3 >= (int64_t)INT32_MAX)
            return VRT_E_BAD_SHAPE;
    }
    if (m->env_sampler == 1) {
        if (!m->env_quadtree) return VRT_E_NULL_POINTER;
        if (m->env_levels < 1 || m->env_levels > 14) return VRT_E_BAD_SHAPE;
    }
    if (m->emission_is_grid) {
        st = to_dgrid(m->emission_grid, 0, M.emission_grid);
        if (st) return st;
        if (M.emission_grid.C != 1 && M.emission_grid.C != 3) return VRT_E_BAD_SHAPE;
    }
    if (m->majorant_mode == 1) {
        if (!m->maj_grid) return VRT_E_NULL_POINTER;
        if (m->maj_dims[0] < 1 || m->maj_dims[1] < 1 || m->maj_dims[2] < 1) return VRT_E_BAD_SHAPE;
        if (!finite3(m->maj_scale)) return VRT_E_NONFINITE;
    } else if (m->majorant_mode != 0) {
        return VRT_E_INVALID_ARGUMENT;
    }
    M.bmin = mk3(m->bmin); M.bmax = mk3(m->bmax); M.inv_bsize = mk3(m->inv_bsize);
    M.box_min = mk3(m->box_min); M.box_max = mk3(m->box_max);
    M.albedo_is_grid = m->albedo_is_grid ? 1 : 0;
    M.albedo_const = mk3(m->albedo_const); M.emission = mk3(m->emission); M.env = mk3(m->env);
    M.has_sun = m->has_sun ? 1 : 0;
    M.sun_dir = mk3(m->sun_dir); M.sun_L = mk3(m->sun_radiance);
    M.phase_mode = m->phase_mode; M.g = m->phase_g;
    M.maj_mode = m->majorant_mode; M.gmaj = m->global_majorant;
    M.maj = m->maj_grid;
    M.Mx = m->maj_dims[0]; M.My = m->maj_dims[1]; M.Mz = m->maj_dims[2];
    M.maj_scale = mk3(m->maj_scale);
    M.tr_mode = m->transmittance_mode;
    M.max_bounces = m->max_bounces;
    M.ds_eps = m->ds_epsilon;
    M.ds_compat = m->ds_compat;
    M.exitance_mode = m->exitance_mode;
    M.emission_is_grid = m->emission_is_grid ? 1 : 0;
    M.env_mode = m->env_mode;
    M.env_img = m->env_image;
    M.env_h = m->env_hw[0];
    M.env_w = m->env_hw[1];
    M.env_sampler = m->env_sampler;
    M.env_qt = m->env_quadtree;
    M.env_levels = m->env_levels;
    return VRT_OK;
}

static int to_dcamera(const vrt_camera* c, DCamera& C) {
    if (!c) return VRT_E_NULL_POINTER;
    if (!c->poses) return VRT_E_NULL_POINTER;
    if (c->views < 1 || c->height < 1 || c->width < 1) return VRT_E_BAD_SHAPE;
    if (!std::isfinite(c->fov) || !std::isfinite(c->znear) || c->fov <= 0.0f || c->znear <= 0.0f) return VRT_E_INVALID_ARGUMENT;
    if (c->sensors && c->n_sensors < 1) return VRT_E_BAD_SHAPE;
    C.poses = c->poses;
    C.views = c->views; C.height = c->height; C.width = c->width;
    C.fov = c->fov; C.znear = c->znear; C.jittered = c->jittered ? 1 : 0;
    C.sensors = reinterpret_cast<const long long*>(c->sensors);
    return VRT_OK;
}

// pixels of a capture: every pixel of every view, or the sensors batch
static long long capture_pixels(const vrt_camera* c) {
    return c->sensors ? (long long)c->n_sensors : (long long)c->views * c->height * c->width;
}

static int check_ctx(vrt_context* ctx) {
    if (!ctx || !ctx->scratch) return VRT_E_NULL_POINTER;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return VRT_E_CUDA;
    if (dev != ctx->device) return VRT_E_INVALID_ARGUMENT;
    return VRT_OK;
}

static bool aligned8(const void* p) { return ((uintptr_t)p & 7u) == 0; }

}  // namespace vrt

using namespace vrt;

extern "C" {

int32_t vrt_version(void) { return 1; }

int64_t vrt_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int vrt_gather_peak(const void* buffer, int64_t bytes, int64_t threads, int32_t per_thread, uint32_t seed,
                    uint32_t* sink, void* stream) {
    if (!buffer || !sink) return VRT_E_NULL_POINTER;
    if (bytes < 64 || threads < 256 || per_thread < 4 || (per_thread & 3) || ((uintptr_t)buffer & 31u))
        return VRT_E_INVALID_ARGUMENT;
    const unsigned long long sectors = (unsigned long long)bytes / 32ull;
    if (sectors > (1ull << 32)) return VRT_E_BAD_SHAPE;
    const int blocks = (int)(threads / 256);
    k_gather_peak<<<blocks, 256, 0, (cudaStream_t)stream>>>(static_cast<const uint4*>(buffer), sectors, per_thread,
                                                            seed, sink);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_atomic_peak(float* buffer, int64_t n, int64_t threads, int32_t per_thread, int32_t pairs, uint32_t seed,
                    void* stream) {
    if (!buffer) return VRT_E_NULL_POINTER;
    if (n < 2 || threads < 256 || per_thread < 4 || (per_thread & 3) || ((uintptr_t)buffer & 7u))
        return VRT_E_INVALID_ARGUMENT;
    if ((unsigned long long)n > (1ull << 32)) return VRT_E_BAD_SHAPE;
    const int blocks = (int)(threads / 256);
    k_atomic_peak<<<blocks, 256, 0, (cudaStream_t)stream>>>(buffer, (unsigned long long)n, per_thread, pairs ? 1 : 0,
                                                            seed);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_set_wave_batch_limit(vrt_context* ctx, int64_t items) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (items < 0) return VRT_E_BAD_SHAPE;
    ctx->batch_limit = (unsigned long long)items;
    return VRT_OK;
}

int vrt_set_collision_log_limit(vrt_context* ctx, int64_t events) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (events < 0) return VRT_E_BAD_SHAPE;
    ctx->log_limit = (unsigned long long)events;
    return VRT_OK;
}

void vrt_set_kernel_timing(int32_t on) {
    KernelTiming& t = timing();
    std::lock_guard<std::mutex> lock(t.mu);
    t.on = on != 0;
}

int vrt_kernel_stats(vrt_context* ctx, void* stream, vrt_kernel_stat* out) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (!out) return VRT_E_NULL_POINTER;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaStreamSynchronize(s) != cudaSuccess) return launch_status(cudaGetLastError());
    unsigned long long k[VRT_K_COUNT][5];
    static_assert(sizeof(k) == sizeof(DScratch::kstat), "one counter slot per kernel");
    if (cudaMemcpy(k, ctx->scratch->kstat, sizeof(k), cudaMemcpyDeviceToHost) != cudaSuccess) return VRT_E_CUDA;
    if (cudaMemset(ctx->scratch->kstat, 0, sizeof(k)) != cudaSuccess) return VRT_E_CUDA;
    KernelTiming& t = timing();
    std::lock_guard<std::mutex> lock(t.mu);
    double ms[VRT_K_COUNT] = {};
    for (const auto& p : t.pending) {
        float e = 0.0f;
        if (cudaEventSynchronize(p.e1) == cudaSuccess && cudaEventElapsedTime(&e, p.e0, p.e1) == cudaSuccess)
            ms[p.kid] += e;
        else
            cudaGetLastError();
        t.pool.push_back(p.e0);
        t.pool.push_back(p.e1);
    }
    t.pending.clear();
    for (int i = 0; i < VRT_K_COUNT; ++i) {
        out[i].launches = t.launches[i];
        out[i].ms = ms[i];
        out[i].steps = (int64_t)k[i][0];
        out[i].lookups = (int64_t)k[i][1];
        out[i].reds = (int64_t)k[i][2];
        out[i].albedo_lookups = (int64_t)k[i][3];
        out[i].log_bytes = (int64_t)k[i][4];
        t.launches[i] = 0;
    }
    return VRT_OK;
}

const char* vrt_status_string(int32_t s) {
    switch (s) {
        case VRT_OK: return "ok";
        case VRT_E_INVALID_ARGUMENT: return "invalid argument";
        case VRT_E_NULL_POINTER: return "null pointer";
        case VRT_E_BAD_SHAPE: return "bad shape or strides";
        case VRT_E_ITER_CAP: return "device loop iteration cap reached";
        case VRT_E_NONFINITE: return "non-finite value";
        case VRT_E_CUDA: return "CUDA error";
        case VRT_E_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

int vrt_context_create(int32_t device, vrt_context** out) {
    if (!out) return VRT_E_NULL_POINTER;
    *out = nullptr;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return VRT_E_CUDA;
    if (device != cur) return VRT_E_INVALID_ARGUMENT;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return VRT_E_CUDA;
    vrt_context* ctx = new vrt_context;
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    ctx->scratch = nullptr;
    ctx->wave = nullptr;
    ctx->wave_bytes = 0;
    ctx->log_limit = 0;
    ctx->batch_limit = 0;
    if (cudaMalloc(&ctx->scratch, sizeof(DScratch)) != cudaSuccess) { delete ctx; return VRT_E_CUDA; }
    if (cudaMemset(ctx->scratch, 0, sizeof(DScratch)) != cudaSuccess) { cudaFree(ctx->scratch); delete ctx; return VRT_E_CUDA; }
    *out = ctx;
    return VRT_OK;
}

int vrt_context_destroy(vrt_context* ctx) {
    if (!ctx) return VRT_E_NULL_POINTER;
    cudaError_t e = cudaFree(ctx->scratch);
    if (ctx->wave) cudaFree(ctx->wave);
    delete ctx;
    return e == cudaSuccess ? VRT_OK : VRT_E_CUDA;
}

int vrt_context_sync(vrt_context* ctx, void* stream, vrt_counters* out) {
    int st = check_ctx(ctx);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaStreamSynchronize(s) != cudaSuccess) return launch_status(cudaGetLastError());
    DScratch h;
    if (cudaMemcpyAsync(&h, ctx->scratch, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess) return VRT_E_CUDA;
    // the per-kernel slots (kstat) stay: vrt_kernel_stats reads and clears them
    if (cudaMemsetAsync(ctx->scratch, 0, offsetof(DScratch, kstat), s) != cudaSuccess) return VRT_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return VRT_E_CUDA;
    if (out) {
        out->paths = (int64_t)h.paths;
        out->vertices = (int64_t)h.vertices;
        out->steps = (int64_t)h.steps;
        out->lookups = (int64_t)h.lookups;
        out->reds = (int64_t)h.reds;
        out->albedo_lookups = (int64_t)h.albedo;
        out->status = (int64_t)h.status;
        out->detail = (int64_t)h.detail;
    }
    for (int code = 1; code < 8; ++code)
        if (h.status & (1u << code)) return code;
    return VRT_OK;
}

int vrt_ray_box(const float* rays, int64_t n, const float bmin[3], const float bmax[3], float* out, void* stream) {
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!rays || !bmin || !bmax || !out) return VRT_E_NULL_POINTER;
    k_ray_box<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(rays, n, mk3(bmin), mk3(bmax), out);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_grid3d_fw(const vrt_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, int64_t n,
                  float* out, void* stream) {
    if (!g || !bmin || !inv_bsize) return VRT_E_NULL_POINTER;
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0) return VRT_OK;
    if (!x || !out) return VRT_E_NULL_POINTER;
    DGrid G;
    int st = to_dgrid(*g, 0, G);
    if (st) return st;
    k_grid_fw<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(G, mk3(bmin), mk3(inv_bsize), x, n, out);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_grid3d_bw(const vrt_grid* g, const float bmin[3], const float inv_bsize[3], const float* x, const float* dout,
                  int64_t n, void* stream) {
    if (!g || !bmin || !inv_bsize) return VRT_E_NULL_POINTER;
    if (n < 0) return VRT_E_BAD_SHAPE;
    if (n == 0 || !g->grad) return VRT_OK;
    if (!x || !dout) return VRT_E_NULL_POINTER;
    DGrid G;
    int st = to_dgrid(*g, 0, G);
    if (st) return st;
    k_grid_bw<<<blocks_for(n), 256, 0, (cudaStream_t)stream>>>(G, mk3(bmin), mk3(inv_bsize), x, dout, n);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_majorant_build(const vrt_grid* sigma, int32_t brick, float* out, int32_t dims_out[3], void* stream) {
    if (!sigma || !dims_out) return VRT_E_NULL_POINTER;
    if (brick < 1) return VRT_E_INVALID_ARGUMENT;
    DGrid G;
    int st = to_dgrid(*sigma, 0, G);
    if (st) return st;
    int M[3] = {(G.W - 1 + brick - 1) / brick, (G.H - 1 + brick - 1) / brick, (G.D - 1 + brick - 1) / brick};
    dims_out[0] = M[0]; dims_out[1] = M[1]; dims_out[2] = M[2];
    if (!out) return VRT_OK;
    int64_t total = (int64_t)M[0] * M[1] * M[2];
    k_majorant_build<<<blocks_for(total * 32), 256, 0, (cudaStream_t)stream>>>(G, brick, M[0], M[1], M[2], out);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int vrt_transmittance_fw(vrt_context* ctx, const vrt_medium* m, int32_t mode, const float* rays, int64_t n,
                         uint64_t seed, float* T, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (mode < 0 || mode > 5) return VRT_E_INVALID_ARGUMENT;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (n == 0) return VRT_OK;
    if (!rays || !T) return VRT_E_NULL_POINTER;
    if (!aligned8(rays)) return VRT_E_INVALID_ARGUMENT;
    return launch_transmittance_fw(M, mode, rays, n, seed, T, ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
}

int vrt_transmittance_bw(vrt_context* ctx, const vrt_medium* m, int32_t mode, const float* rays, int64_t n,
                         uint64_t seed, const float* dL_dT, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (mode < 0 || mode > 5) return VRT_E_INVALID_ARGUMENT;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    // GRT / GDT have no backward (the reference's maps define none): no gradient
    if (n == 0 || !M.sigma.grad || mode >= 4) return VRT_OK;
    if (!rays || !dL_dT) return VRT_E_NULL_POINTER;
    if (!aligned8(rays)) return VRT_E_INVALID_ARGUMENT;
    float* tmp = nullptr;  // the DDA adjoint's dL/dtau per ray, in the context's work buffer
    if (mode == 2 || mode == 3) {
        if ((st = ensure_wave_buffer(ctx, (size_t)n * sizeof(float)))) return st;
        tmp = static_cast<float*>(ctx->wave);
    }
    return launch_transmittance_bw(M, mode, rays, n, seed, dL_dT, tmp, ctx->scratch, ctx->num_sms,
                                   (cudaStream_t)stream);
}

int vrt_collision_sample_fw(vrt_context* ctx, const vrt_medium* m, const float* rays, int64_t n, uint64_t seed,
                            float* out, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (n == 0) return VRT_OK;
    if (!rays || !out) return VRT_E_NULL_POINTER;
    return launch_collision_sample(M, rays, n, seed, out, nullptr, ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
}

int vrt_collision_sample_bw(vrt_context* ctx, const vrt_medium* m, const float* rays, int64_t n, uint64_t seed,
                            const float* dL_dout, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (n == 0 || !M.sigma.grad) return VRT_OK;
    if (!rays || !dL_dout) return VRT_E_NULL_POINTER;
    return launch_collision_sample(M, rays, n, seed, nullptr, dL_dout, ctx->scratch, ctx->num_sms,
                                   (cudaStream_t)stream);
}

int vrt_radiance_fw(vrt_context* ctx, const vrt_medium* m, int32_t integrator, const float* rays, int64_t n,
                    uint64_t seed, float* R, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (integrator < 0 || integrator > VRT_PI_DDA_COLLISION) return VRT_E_INVALID_ARGUMENT;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (n == 0) return VRT_OK;
    if (!rays || !R) return VRT_E_NULL_POINTER;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    S.is_camera = 0;
    S.rays = rays;
    if (is_collision(integrator))
        return launch_collision_fw(M, integrator, S, (uint64_t)n, seed, R, 1.0f, ctx->scratch, ctx->num_sms,
                                   (cudaStream_t)stream);
    if (use_wave(M, integrator)) {  // the wavefront accumulates: clear R first
        cudaError_t e = cudaMemsetAsync(R, 0, sizeof(float) * 3 * (size_t)n, (cudaStream_t)stream);
        if (e != cudaSuccess) return launch_status(e);
        return launch_wave_fw(ctx, M, S, (uint64_t)n, seed, R, 1.0f, (cudaStream_t)stream);
    }
    return launch_radiance_fw(M, integrator, S, (uint64_t)n, seed, R, 1.0f, ctx->scratch, ctx->num_sms,
                              (cudaStream_t)stream);
}

int vrt_radiance_bw(vrt_context* ctx, const vrt_medium* m, int32_t bw_mode, const float* rays, int64_t n,
                    uint64_t seed, const float* dL_dR, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (bw_mode < 0 || bw_mode > VRT_BW_DDA_COLLISION) return VRT_E_INVALID_ARGUMENT;
    if (n < 0) return VRT_E_BAD_SHAPE;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (n == 0) return VRT_OK;
    if (!rays || !dL_dR) return VRT_E_NULL_POINTER;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    S.is_camera = 0;
    S.rays = rays;
    if (bw_mode >= VRT_BW_MC_COLLISION)
        return launch_collision_bw(M, collision_of(bw_mode), S, (uint64_t)n, seed, dL_dR, 1.0f, ctx->scratch,
                                   ctx->num_sms, (cudaStream_t)stream);
    if (use_wave_bw(M, bw_mode)) return launch_wave_ds_bw(ctx, M, S, (uint64_t)n, seed, dL_dR, 1.0f, (cudaStream_t)stream);
    if (use_wave_drt(M, bw_mode))
        return launch_wave_drt_bw(ctx, M, bw_mode, S, (uint64_t)n, seed, dL_dR, 1.0f, (cudaStream_t)stream);
    if (use_wave_sps(M, bw_mode))
        return launch_wave_sps_bw(ctx, M, S, (uint64_t)n, seed, dL_dR, 1.0f, (cudaStream_t)stream);
    return launch_radiance_bw(M, bw_mode, S, (uint64_t)n, seed, dL_dR, 1.0f, ctx->scratch, ctx->num_sms,
                              (cudaStream_t)stream);
}

int vrt_capture_fw(vrt_context* ctx, const vrt_medium* m, int32_t integrator, const vrt_camera* cam, int32_t spp,
                   uint64_t seed, float* rgb, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (integrator < 0 || integrator > VRT_PI_DDA_COLLISION) return VRT_E_INVALID_ARGUMENT;
    if (spp < 1) return VRT_E_INVALID_ARGUMENT;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    if ((st = to_dcamera(cam, S.cam))) return st;
    if (!rgb) return VRT_E_NULL_POINTER;
    S.is_camera = 1;
    S.npix = capture_pixels(cam);
    cudaError_t e = cudaMemsetAsync(rgb, 0, sizeof(float) * 3 * S.npix, (cudaStream_t)stream);
    if (e != cudaSuccess) return launch_status(e);
    if (is_collision(integrator))
        return launch_collision_fw(M, integrator, S, (uint64_t)S.npix * (uint64_t)spp, seed, rgb, 1.0f / (float)spp,
                                   ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
    if (use_wave(M, integrator))
        return launch_wave_fw(ctx, M, S, (uint64_t)S.npix * (uint64_t)spp, seed, rgb, 1.0f / (float)spp,
                              (cudaStream_t)stream);
    return launch_radiance_fw(M, integrator, S, (uint64_t)S.npix * (uint64_t)spp, seed, rgb, 1.0f / (float)spp,
                              ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
}

int vrt_capture_bw(vrt_context* ctx, const vrt_medium* m, int32_t bw_mode, const vrt_camera* cam, int32_t spp,
                   uint64_t seed, const float* dL_drgb, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (bw_mode < 0 || bw_mode > VRT_BW_DDA_COLLISION) return VRT_E_INVALID_ARGUMENT;
    if (spp < 1) return VRT_E_INVALID_ARGUMENT;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    if ((st = to_dcamera(cam, S.cam))) return st;
    if (!dL_drgb) return VRT_E_NULL_POINTER;
    S.is_camera = 1;
    S.npix = capture_pixels(cam);
    if (bw_mode >= VRT_BW_MC_COLLISION)
        return launch_collision_bw(M, collision_of(bw_mode), S, (uint64_t)S.npix * (uint64_t)spp, seed, dL_drgb,
                                   (float)spp, ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
    if (use_wave_bw(M, bw_mode))
        return launch_wave_ds_bw(ctx, M, S, (uint64_t)S.npix * (uint64_t)spp, seed, dL_drgb, (float)spp,
                                 (cudaStream_t)stream);
    if (use_wave_drt(M, bw_mode))
        return launch_wave_drt_bw(ctx, M, bw_mode, S, (uint64_t)S.npix * (uint64_t)spp, seed, dL_drgb, (float)spp,
                                  (cudaStream_t)stream);
    if (use_wave_sps(M, bw_mode))
        return launch_wave_sps_bw(ctx, M, S, (uint64_t)S.npix * (uint64_t)spp, seed, dL_drgb, (float)spp,
                                  (cudaStream_t)stream);
    return launch_radiance_bw(M, bw_mode, S, (uint64_t)S.npix * (uint64_t)spp, seed, dL_drgb, (float)spp,
                              ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
}

int vrt_capture_fw_fp64(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, int32_t spp, uint64_t seed,
                        double* rgb, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (spp < 1) return VRT_E_INVALID_ARGUMENT;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    if (M.env_mode != 0 || M.env_sampler != 0 || M.tr_mode > 1) return VRT_E_UNSUPPORTED;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    if ((st = to_dcamera(cam, S.cam))) return st;
    if (!rgb) return VRT_E_NULL_POINTER;
    S.is_camera = 1;
    S.npix = capture_pixels(cam);
    cudaError_t e = cudaMemsetAsync(rgb, 0, sizeof(double) * 3 * S.npix, (cudaStream_t)stream);
    if (e != cudaSuccess) return launch_status(e);
    return launch_capture_fp64(M, S, spp, seed, rgb, ctx->scratch, ctx->num_sms, (cudaStream_t)stream);
}

int vrt_capture_prefix_fw(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, int32_t spp, uint64_t seed,
                          int32_t cut, float* rgb, float* queries, void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (spp < 1 || cut < 0) return VRT_E_INVALID_ARGUMENT;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    if ((st = to_dcamera(cam, S.cam))) return st;
    if (!rgb || !queries) return VRT_E_NULL_POINTER;
    S.is_camera = 1;
    S.npix = capture_pixels(cam);
    const uint64_t n = (uint64_t)S.npix * (uint64_t)spp;
    // the wavefront forward with a cut (its job reserve is bounded by the cut,
    // capped or not); very deep cuts stay on the per-lane state machine
    if (cut <= 4096 && (M.max_bounces <= 0 || M.max_bounces <= 4096))
        return launch_wave_fw(ctx, M, S, n, seed, rgb, 1.0f / (float)spp, (cudaStream_t)stream, cut, queries);
    CacheIO io = {cut, 0, queries, nullptr, nullptr, (long long)n};
    return launch_cache_paths(M, FW_CUT, S, n, seed, rgb, 1.0f / (float)spp, io, ctx->scratch, ctx->num_sms,
                              (cudaStream_t)stream);
}

int vrt_capture_train_samples(vrt_context* ctx, const vrt_medium* m, const vrt_camera* cam, const vrt_cache* c,
                              int32_t cut, int64_t n_paths, uint64_t seed, int32_t rec, float* samples, float* work,
                              void* stream) {
    int st = check_ctx(ctx);
    if (st) return st;
    if (n_paths < 0 || rec < 1 || rec > 8) return VRT_E_INVALID_ARGUMENT;
    if (c && cut < rec) return VRT_E_INVALID_ARGUMENT;
    DMedium M;
    if ((st = to_dmedium(m, M))) return st;
    PathSrc S;
    std::memset(&S, 0, sizeof(S));
    if ((st = to_dcamera(cam, S.cam))) return st;
    if (!samples || !work) return VRT_E_NULL_POINTER;
    S.is_camera = 1;
    S.npix = capture_pixels(cam);
    if (S.npix >= (1ll << 32)) return VRT_E_BAD_SHAPE;
    if (n_paths == 0) return VRT_OK;
    float* pR = work;
    float* q = work + 3 * n_paths;
    CacheIO io = {c ? cut : -1, rec, q, samples, pR, (long long)n_paths};
    cudaStream_t s = (cudaStream_t)stream;
    if ((st = launch_cache_paths(M, FW_TRAIN, S, (uint64_t)n_paths, seed, nullptr, 0.0f, io, ctx->scratch,
                                 ctx->num_sms, s)))
        return st;
    if (c && (st = vrt_cache_resolve(c, q, n_paths, n_paths, 1.0f, pR, stream))) return st;
    return launch_cache_targets(samples, pR, n_paths, rec, s);
}

}  // extern "C"
