// vrt_transmittance.cu -- transmittance maps evaluated on rays [n, 6] (sm_100a).
//
// One thread per ray; ray i draws from Philox path id i.  These are the
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
        if (MODE == 2) v = transmittance_dda<false>(M, x, w, tl);
        else if (MODE == 3) v = transmittance_dda<true>(M, x, w, tl);
        else {
            Rng path;
            path.init(seed, (uint64_t)i, 0);
            Rng rng = path.fork();  // as the dispatch of a path integrator would
            if (MODE == 0) v = transmittance_rt(M, rng, x, w, tl, &sc->status);
            else if (MODE == 1) v = transmittance_dt(M, rng, x, w, tl, &sc->status);
            else v = transmittance_grid_tracking<MODE == 5>(M, rng, x, w, tl, &sc->status);
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
        if (MODE == 2) transmittance_dda_bw<false>(M, x, w, g, tl);
        else if (MODE == 3) transmittance_dda_bw<true>(M, x, w, g, tl);
        else {
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

static int grid_for(int64_t n) {
    int64_t b = (n + 255) / 256;
    return (int)(b < 65535 * 8 ? (b < 1 ? 1 : b) : 65535 * 8);
}

int launch_transmittance_fw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed, float* T,
                            DScratch* scratch, cudaStream_t stream) {
    if (n == 0) return 0;
    int g = grid_for(n);
    switch (mode) {
        case 0: k_transmittance_fw<0><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
        case 1: k_transmittance_fw<1><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
        case 2: k_transmittance_fw<2><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
        case 3: k_transmittance_fw<3><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
        case 4: k_transmittance_fw<4><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
        default: k_transmittance_fw<5><<<g, 256, 0, stream>>>(M, rays, n, seed, T, scratch); break;
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_transmittance_bw(const DMedium& M, int mode, const float* rays, int64_t n, uint64_t seed,
                            const float* dL_dT, DScratch* scratch, cudaStream_t stream) {
    if (n == 0) return 0;
    int g = grid_for(n);
    switch (mode) {
        case 0: k_transmittance_bw<0><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
        case 1: k_transmittance_bw<1><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
        case 2: k_transmittance_bw<2><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
        default: k_transmittance_bw<3><<<g, 256, 0, stream>>>(M, rays, n, seed, dL_dT, scratch); break;
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
