// vrt_transmittance.cu -- transmittance maps evaluated on rays [n, 6] (sm_100a).
//
// GRT and the RT / DT adjoints: one thread per ray; the DDA, GDT, RT and DT
// forwards: persistent lanes refilled ray by ray.  Ray i draws from Philox
// path id i.  These are the
// operator forms of GridDDATransmittance / RatiotrackingTransmittance /
// DeltatrackingTransmittance, GridRatiotrackingTransmittance and
// GridDeltatrackingTransmittance (include/maps/transmittance_{dda,rt,dt,grt,gdt}.h).
#include <cuda_runtime.h>

#include "vrt_internal.h"
#include "vrt_tracking.cuh"

namespace vrt {

__device__ __forceinline__ void warp_tally(DScratch* sc, uint32_t count, const Tally& tl) {
    unsigned long long p = count, s = tl.steps, l = tl.lookups, r = tl.reds;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
        l += __shfl_down_sync(0xffffffffu, l, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sc->paths, p);
        atomicAdd(&sc->steps, s);
        atomicAdd(&sc->lookups, l);
        atomicAdd(&sc->reds, r);
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_transmittance_fw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                           uint64_t seed, float* __restrict__ T, DScratch* sc) {
    uint32_t count = 0;
    Tally tl;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2* r2 = reinterpret_cast<const float2*>(rays + 6 * i);  // rows are 8-byte aligned
        float2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2);
        float3 x = make_float3(a.x, a.y, b.x), w = make_float3(b.y, c.x, c.y);
        float v;
        {
            Rng path;
            path.init(seed, (uint64_t)i, 0);
            Rng rng = path.fork();  // as the dispatch of a path integrator would
            if (MODE == 0) v = transmittance_rt(M, rng, x, w, tl, &sc->status);
            else if (MODE == 1) v = transmittance_dt(M, rng, x, w, tl, &sc->status);
            else v = transmittance_grid_tracking<false>(M, rng, x, w, tl, &sc->status);
        }
        T[i] = v;
        ++count;
    }
    warp_tally(sc, count, tl);
}

template <int MODE>
__global__ void __launch_bounds__(256) k_transmittance_bw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                           uint64_t seed, const float* __restrict__ dL_dT,
                                                           DScratch* sc) {
    uint32_t count = 0;
    Tally tl;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2* r2 = reinterpret_cast<const float2*>(rays + 6 * i);
        float2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2);
        float3 x = make_float3(a.x, a.y, b.x), w = make_float3(b.y, c.x, c.y);
        float g = __ldg(dL_dT + i);
        {
            Rng path;
            path.init(seed, (uint64_t)i, 0);
            Rng rng = path.fork();
            if (MODE == 0) transmittance_rt_bw(M, rng, x, w, g, tl, &sc->status);
            else transmittance_dt_bw(M, rng, x, w, g, tl, &sc->status);
        }
        ++count;
    }
    warp_tally(sc, count, tl);
}

// The DDA modes as persistent lanes: a lane takes the next ray as soon as its
// march ends (one atomic per warp refill, from the scratch's work counter), so
// the short and missing rays of a warp do not wait for its longest (one ray
// per thread kept 7.7 of 32 lanes active).  A ray's arithmetic is
// transmittance_dda's, cell for cell; at most kCells cells per lane between
// refills.
constexpr int kCells = 8;

__device__ __forceinline__ bool take_ray(DScratch* sc, int64_t n, bool want_ray, int64_t& i) {
    const unsigned want = __ballot_sync(0xffffffffu, want_ray);
    if (!want) return false;
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(want) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!want_ray) return false;
    i = (int64_t)(base + __popc(want & ((1u << lane) - 1u)));
    return true;
}
__device__ __forceinline__ void load_ray(const float* rays, int64_t i, float3& x, float3& w) {
    const float2* r2 = reinterpret_cast<const float2*>(rays + 6 * i);  // rows are 8-byte aligned
    const float2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2);
    x = make_float3(a.x, a.y, b.x);
    w = make_float3(b.y, c.x, c.y);
}

// BW = false: T of every ray into out.  BW = true, the adjoint's first march:
// dL/dtau = -dL/dT T into out (0 for a ray with dL/dT = 0, which it skips,
// and for a miss), for k_dda_scatter.
template <bool EXACT, bool BW>
__global__ void __launch_bounds__(256) k_dda_fw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                const float* __restrict__ dL_dT, float* __restrict__ out,
                                                DScratch* sc) {
    DDA q;
    float acc = 0.0f, comp = 0.0f, ct = 0.0f, stop = 0.0f, g = 0.0f;
    int it = 0;
    int64_t ray = -1;
    bool exhausted = false;
    uint32_t count = 0;
    Tally tl;
    while (true) {
        int64_t i;
        if (take_ray(sc, n, ray < 0 && !exhausted, i)) {
            if (i >= n) {
                exhausted = true;
            } else {
                float3 x, w;
                load_ray(rays, i, x, w);
                if (BW) g = __ldg(dL_dT + i);
                else ++count;
                if ((BW && g == 0.0f) || !q.init(M, x, w)) {
                    out[i] = BW ? 0.0f : 1.0f;  // no gradient, or a miss
                } else {
                    q.load_all(M.sigma);
                    acc = 0.0f;
                    comp = 0.0f;
                    ct = 0.0f;
                    it = 0;
                    stop = q.tau_stop<EXACT>();
                    ray = i;
                }
            }
        }
        if (__all_sync(0xffffffffu, ray < 0 && exhausted)) break;
        if (ray >= 0) {
            for (int c = 0; c < kCells; ++c) {
                if (!(ct < stop && it < kStepCap)) {
                    out[ray] = BW ? -g * expf(-acc) : expf(-acc);
                    ray = -1;
                    break;
                }
                q.tau_cell<EXACT>(M.sigma, acc, comp, ct);
                ++tl.steps;
                ++tl.lookups;
                ++it;
            }
        }
    }
    warp_tally(sc, count, tl);
}

// GridDeltatracking (DELTA) on the same refilled lanes, one cell (its
// minorant part and its tracking steps) per iteration; ray i draws from fork 0
// of path i's stream, as transmittance_grid_tracking does.
template <bool DELTA>
__global__ void __launch_bounds__(256) k_grid_tracking_fw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                          uint64_t seed, float* __restrict__ out, DScratch* sc) {
    DDA q;
    Rng rng;
    float T = 1.0f, ct = 0.0f, stop = 0.0f;
    int it = 0;
    int64_t ray = -1;
    bool exhausted = false;
    uint32_t count = 0;
    Tally tl;
    while (true) {
        int64_t i;
        if (take_ray(sc, n, ray < 0 && !exhausted, i)) {
            if (i >= n) {
                exhausted = true;
            } else {
                float3 x, w;
                load_ray(rays, i, x, w);
                ++count;
                if (!q.init(M, x, w)) {
                    out[i] = 1.0f;  // a miss
                } else {
                    Rng path;
                    path.init(seed, (uint64_t)i, 0);
                    rng = path.fork();  // as the dispatch of a path integrator would
                    q.load_all(M.sigma);
                    T = 1.0f;
                    ct = 0.0f;
                    it = 0;
                    stop = q.d - 0.0001f;
                    ray = i;
                }
            }
        }
        if (__all_sync(0xffffffffu, ray < 0 && exhausted)) break;
        if (ray >= 0) {
            bool done = !(ct < stop);
            if (!done) {
                if (++it > kStepCap) {
                    raise_status(&sc->status, 4);
                    done = true;
                } else {
                    done = !grid_tracking_cell<DELTA>(M, q, rng, T, ct, it, tl, &sc->status);
                }
            }
            if (done) {
                out[ray] = T;
                ray = -1;
            }
        }
    }
    warp_tally(sc, count, tl);
}

// RatiotrackingTransmittance / DeltatrackingTransmittance (DELTA) on the
// refilled lanes, at most kTrackSteps tracking steps (crossings or
// collisions) per lane between refills; ray i draws from fork 0 of path i's
// stream, as transmittance_rt / _dt do.
constexpr int kTrackSteps = 4;
template <bool DELTA>
__global__ void __launch_bounds__(256) k_track_fw(DMedium M, const float* __restrict__ rays, int64_t n, uint64_t seed,
                                                  float* __restrict__ out, DScratch* sc) {
    Flight ff;
    Rng rng;
    float3 x = make_float3(0.0f, 0.0f, 0.0f), w = x;
    float d = 0.0f, T = 1.0f;
    int it = 0;
    int64_t ray = -1;
    bool exhausted = false;
    uint32_t count = 0;
    Tally tl;
    while (true) {
        int64_t i;
        if (take_ray(sc, n, ray < 0 && !exhausted, i)) {
            if (i >= n) {
                exhausted = true;
            } else {
                float3 x0;
                load_ray(rays, i, x0, w);
                ++count;
                float tMin, tMax;
                if (!boundary(M, x0, w, tMin, tMax)) {
                    out[i] = 1.0f;  // a miss
                } else {
                    Rng path;
                    path.init(seed, (uint64_t)i, 0);
                    rng = path.fork();  // as the dispatch of a path integrator would
                    x = x0 + w * tMin;
                    d = tMax - tMin;
                    ff = Flight();
                    T = 1.0f;
                    it = 0;
                    ray = i;
                }
            }
        }
        if (__all_sync(0xffffffffu, ray < 0 && exhausted)) break;
        if (ray >= 0) {
            for (int c = 0; c < kTrackSteps; ++c) {
                if (it >= kStepCap) {
                    raise_status(&sc->status, 4);
                    out[ray] = DELTA ? 1.0f : T;
                    ray = -1;
                    break;
                }
                ++it;
                if (DELTA) {
                    const int r = dt_step(M, rng, ff, x, w, d, tl);
                    if (r) {
                        out[ray] = r == 1 ? 1.0f : 0.0f;
                        ray = -1;
                        break;
                    }
                } else if (rt_step(M, rng, ff, x, w, d, T, tl)) {
                    out[ray] = T;
                    ray = -1;
                    break;
                }
            }
        }
    }
    warp_tally(sc, count, tl);
}

// The adjoint's second march (transmittance_dda_bw after its tau): rays with
// dL/dtau != 0 scatter from the segment's start.
template <bool EXACT>
__global__ void __launch_bounds__(256) k_dda_scatter(DMedium M, const float* __restrict__ rays, int64_t n,
                                                     const float* __restrict__ dL_dtau, DScratch* sc) {
    DDA q;
    float ct = 0.0f, stop = 0.0f, g = 0.0f;
    float gacc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) gacc[k] = 0.0f;
    int it = 0;
    bool busy = false, exhausted = false;
    uint32_t count = 0;
    Tally tl;
    while (true) {
        int64_t i;
        if (take_ray(sc, n, !busy && !exhausted, i)) {
            if (i >= n) {
                exhausted = true;
            } else {
                ++count;
                g = __ldg(dL_dtau + i);
                float3 x, w;
                load_ray(rays, i, x, w);
                if (g != 0.0f && q.init(M, x, w)) {
#pragma unroll
                    for (int k = 0; k < 8; ++k) gacc[k] = 0.0f;
                    ct = 0.0f;
                    it = 0;
                    stop = q.tau_stop<EXACT>();
                    busy = true;
                }
            }
        }
        if (__all_sync(0xffffffffu, !busy && exhausted)) break;
        if (busy) {
            for (int c = 0; c < kCells; ++c) {
                if (!(ct < stop && it < kStepCap)) {
                    tl.reds += 4;
                    q.scatter_end(M.sigma, gacc);
                    busy = false;
                    break;
                }
                q.scatter_cell<EXACT>(M.sigma, g, gacc, ct);
                tl.reds += 4;
                ++it;
            }
        }
    }
    warp_tally(sc, count, tl);
}

static int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 65535 * 8 ? (b < 1 ? 1 : b) : 65535 * 8);
}

// persistent blocks for the DDA kernels (num_sms < 1: asked of the device)
static int dda_blocks(const void* kernel, int num_sms, int64_t n) {
    if (num_sms < 1) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || num_sms < 1)
            num_sms = 1;
    }
    int b = persistent_blocks(kernel, 256, num_sms);
    const int64_t need = (n + 255) / 256;
    return (int64_t)b > need ? (int)need : b;
}

int launch_transmittance_fw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed, float* T,
                            DScratch* scratch, int num_sms, cudaStream_t stream) {
    if (n == 0) return 0;
    if (mode == 2 || mode == 3) {
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        if (mode == 2)
            k_dda_fw<false, false><<<dda_blocks((const void*)k_dda_fw<false, false>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, nullptr, T, scratch);
        else
            k_dda_fw<true, false><<<dda_blocks((const void*)k_dda_fw<true, false>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, nullptr, T, scratch);
        count_launches(1);
        return launch_status(cudaGetLastError());
    }
    if (mode == 5) {  // GDT: rays end at their first collision, so lengths vary and refilling pays
        // (GRT walks every ray to its end: one ray per thread was faster, 8.6 against 9.9 ms)
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        k_grid_tracking_fw<true><<<dda_blocks((const void*)k_grid_tracking_fw<true>, num_sms, n), 256, 0, stream>>>(
            M, rays, n, seed, T, scratch);
        count_launches(1);
        return launch_status(cudaGetLastError());
    }
    if (mode == 0 || mode == 1) {
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        if (mode == 0)
            k_track_fw<false><<<dda_blocks((const void*)k_track_fw<false>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, seed, T, scratch);
        else
            k_track_fw<true><<<dda_blocks((const void*)k_track_fw<true>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, seed, T, scratch);
        count_launches(1);
        return launch_status(cudaGetLastError());
    }
    int g = grid_for(n);
    k_transmittance_fw<4><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_transmittance_bw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed,
                            const float* dL_dT, float* tmp, DScratch* scratch, int num_sms, cudaStream_t stream) {
    if (n == 0) return 0;
    if (mode == 2 || mode == 3) {  // the tau march into tmp (dL/dtau per ray), then the scatter march
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        if (mode == 2)
            k_dda_fw<false, true><<<dda_blocks((const void*)k_dda_fw<false, true>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, dL_dT, tmp, scratch);
        else
            k_dda_fw<true, true><<<dda_blocks((const void*)k_dda_fw<true, true>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, dL_dT, tmp, scratch);
        if ((e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        if (mode == 2)
            k_dda_scatter<false><<<dda_blocks((const void*)k_dda_scatter<false>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, tmp, scratch);
        else
            k_dda_scatter<true><<<dda_blocks((const void*)k_dda_scatter<true>, num_sms, n), 256, 0, stream>>>(
                M, rays, n, tmp, scratch);
        count_launches(2);
        return launch_status(cudaGetLastError());
    }
    int g = grid_for(n);
    switch (mode) {
        case 0: k_transmittance_bw<0><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
        default: k_transmittance_bw<1><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
