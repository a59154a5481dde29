// vrt_wave.cu -- wavefront form of the NEE path integrator (sm_100a).
//
// The forward NEE integrator (include/vr_path_integrator_NEE.h:1-66, plus the
// directional light and the bounce cap) split in two coherent kernels:
//
//   k_walk_fw    persistent; every lane walks one path's primary segments
//                (delta tracking over the majorant bricks), handles its real
//                collisions (albedo, emission, environment direction, phase
//                sampling) and, instead of tracing the shadow rays, appends
//                them to a job buffer -- position, direction, the weight the
//                shadow transmittance multiplies, and the (path, fork) key of
//                the ray's random stream.  Slots are reserved with one atomic
//                per warp (warp prefix sum of the lanes' job counts).
//   k_shadow_fw  one shadow job per thread: transmittance with the job's own
//                Philox fork, then out[pixel] += weight * T.
//
// A shadow ray's estimate never feeds back into its path (the path only adds
// W * T * L * phase to its estimate), so the split changes no value: the path
// consumes exactly the draws of the sequential definition, and shadow j of
// path p draws from fork j of p's stream in both forms.  Only the order of the
// floating-point sums into a pixel differs.
//
// The job buffer is bounded: a warp takes new paths only while the job count
// plus the worst case of every lane of the launch (1 + lights x max_bounces
// jobs per path) fits, and the host repeats walk + shadow rounds until every
// path is done.  Used for capped NEE paths; the persistent state machine of
// vrt_path.cu serves uncapped ones.
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include "vrt_tracking.cuh"

namespace vrt {

namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kPathCap = 1 << 26;  // free-flight steps of one path before VRT_E_ITER_CAP

// 48 bytes: position, direction, weight, key = pid << 16 | fork
struct ShadowJob {
    float4 a, b, c;
};

__device__ __forceinline__ void put_job(ShadowJob* J, unsigned long long slot, float3 x, float3 d, float3 wt,
                                        unsigned long long key) {
    float4* p = reinterpret_cast<float4*>(J + slot);
    p[0] = make_float4(x.x, x.y, x.z, d.x);
    p[1] = make_float4(d.y, d.z, wt.x, wt.y);
    p[2] = make_float4(wt.z, 0.0f, __uint_as_float((uint32_t)key), __uint_as_float((uint32_t)(key >> 32)));
}

__device__ __forceinline__ unsigned long long job_key(uint64_t pid, uint32_t fork) {
    return ((unsigned long long)pid << 16) | (unsigned long long)(fork & 0xffffu);
}

// Reserves n slots for this lane (all 32 lanes call it): an inclusive warp scan
// of n, one atomicAdd by the last lane, the base broadcast.
__device__ __forceinline__ unsigned long long reserve_slots(unsigned long long* count, int n) {
    const unsigned lane = threadIdx.x & 31u;
    int incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(kAll, incl, o);
        if ((int)lane >= o) incl += v;
    }
    const int total = __shfl_sync(kAll, incl, 31);
    unsigned long long base = 0;
    if (total > 0) {
        if (lane == 31u) base = atomicAdd(count, (unsigned long long)total);
        base = __shfl_sync(kAll, base, 31);
    }
    return base + (unsigned long long)(incl - n);
}

__device__ __forceinline__ void flush_counters(DScratch* sc, uint32_t paths, uint32_t verts, const Tally& tl) {
    unsigned long long p = paths, v = verts, s = tl.steps, l = tl.lookups, a = tl.albedo;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(kAll, p, o);
        v += __shfl_down_sync(kAll, v, o);
        s += __shfl_down_sync(kAll, s, o);
        l += __shfl_down_sync(kAll, l, o);
        a += __shfl_down_sync(kAll, a, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (p) atomicAdd(&sc->paths, p);
        if (v) atomicAdd(&sc->vertices, v);
        if (s) atomicAdd(&sc->steps, s);
        if (l) atomicAdd(&sc->lookups, l);
        if (a) atomicAdd(&sc->albedo, a);
    }
}

__device__ __forceinline__ long long out_index(const PathSrc& S, uint64_t pid) {
    return S.is_camera ? (long long)(pid % (uint64_t)S.npix) : (long long)pid;
}

}  // namespace

struct WaveFw {
    ShadowJob* jobs;
    unsigned long long* count;
    unsigned long long cap, reserve;
};

__global__ void __launch_bounds__(256, 4) k_walk_fw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed, float* out,
                                                  float scale, DScratch* sc, WaveFw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00001f;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f), Rem = f3(0.0f);
    float d = 0.0f;
    int bounces = 0;
    uint64_t pid = 0;
    uint32_t steps_path = 0;
    bool alive = false, exhausted = false;
    uint32_t n_paths_done = 0, n_verts = 0;
    Tally tl;

    while (true) {
        // ---- refill dead lanes while the job buffer has room for the worst case
        int njobs = 0;
        float3 jx = f3(0.0f), jd = f3(0.0f), jw = f3(0.0f), jw2 = f3(0.0f);
        uint32_t jfork = 0;
        unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) {
                const unsigned long long used = *((volatile unsigned long long*)wv.count);
                base = used + wv.reserve > wv.cap ? ~0ull
                                                  : atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
            }
            base = __shfl_sync(kAll, base, leader);
            if (base == ~0ull) {
                exhausted = true;  // no room this round: finish the lanes in flight
            } else if (!alive && !exhausted) {
                const uint64_t p = base + __popc(want & ((1u << lane) - 1u));
                if (p >= n_paths) {
                    exhausted = true;
                } else {
                    // path_integrator_NEE prologue (vr_path_integrator_NEE.h:3-14): the
                    // direct term T(x0, w0) * E becomes a job on fork 0
                    pid = p;
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    if (S.is_camera) {
                        const long long px = (long long)(pid % (uint64_t)S.npix);
                        const long long hw = (long long)S.cam.height * S.cam.width;
                        const int view = (int)(px / hw);
                        const int rem = (int)(px - (long long)view * hw);
                        camera_ray(S.cam, view, rem / S.cam.width, rem % S.cam.width, rng, x0, w0);
                    } else {
                        x0 = ld3(S.rays + 6 * pid);
                        w0 = ld3(S.rays + 6 * pid + 3);
                    }
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    x = x0 + w0 * tMin;
                    w = w0;
                    d = tMax - tMin;
                    W = f3(1.0f);
                    Rem = f3(0.0f);
                    bounces = 0;
                    steps_path = 0;
                    ff = Flight();
                    ++n_paths_done;
                    njobs = 1;
                    jx = x;
                    jd = w;
                    jw = M.env;
                    jfork = rng.ntr++;
                    alive = d > EPS;
                }
            }
        }
        {  // direct-term jobs of the lanes just started
            const unsigned long long slot = reserve_slots(wv.count, njobs);
            if (njobs) put_job(wv.jobs, slot, jx, jd, jw, job_key(pid, jfork));
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        njobs = 0;
        if (alive) {
            // ---- one free flight of the primary segment (vr_path_integrator_NEE.h:20-33);
            // majorant-brick faces are crossed in the inner loop without new draws
            int ev = 0;  // 0 none, 1 collision, 2 escape
            bool need_sigma = false;
            float m = 0.0f, t = 0.0f;
            if (ff.tau < 0.0f) ++tl.steps;
            ff.sample(rng);
            for (int k = 0;; ++k) {
                if (k >= kStepCap) {
                    raise_status(&sc->status, 4);
                    ev = 2;
                    break;
                }
                float md;
                m = gmax(EPS, ff.bk.query(M, x, w, md));
                t = ff.tau / m;
                x = x + w * gmin(t, md);
                if (t > md) {
                    d -= md;
                    ff.cross(m, md);
                    ff.bk.advance(M);
                    if (!(d > EPS)) { ev = 2; break; }
                    continue;
                }
                ff.used();
                if (t > d) ev = 2;
                else need_sigma = true;
                ff.bk.move(t);
                break;
            }
            if (need_sigma) {
                const float s = sigma(M, x, tl);
                if (rng.uniform() >= s / m) {
                    d -= t;
                    if (!(d > EPS)) ev = 2;
                } else {
                    ev = 1;
                }
            }
            if (++steps_path > (uint32_t)kPathCap) {
                raise_status(&sc->status, 4);
                ev = 2;
            }
            if (ev == 1) {  // real collision (vr_path_integrator_NEE.h:41-62)
                ++n_verts;
                const float3 sa = albedo(M, x, tl);
                Rem = Rem + W * (f3(1.0f) - sa) * M.emission;
                W = W * sa;
                float3 wnee;
                const float3 pay = environment_sample(M, rng, wnee);
                njobs = M.has_sun ? 2 : 1;
                jx = x;
                jd = wnee;
                jw = W * pay * phase(M, w, wnee);
                jfork = rng.ntr;
                rng.ntr += (uint32_t)njobs;
                if (M.has_sun) jw2 = W * M.sun_L * phase(M, w, M.sun_dir);
                ++bounces;
                if (M.max_bounces > 0 && bounces >= M.max_bounces) {
                    ev = 2;
                } else {
                    const float3 wo = phase_sample(M, rng, w);
                    if (all_less(W, EPS)) {
                        ev = 2;
                    } else {
                        w = wo;
                        float tMin;
                        boundary(M, x, w, tMin, d);
                        ff = Flight();
                        ev = d > EPS ? 0 : 2;
                    }
                }
            }
            if (ev == 2) {  // the path's estimate is complete (its shadow terms arrive through the jobs)
                if (Rem.x != 0.0f || Rem.y != 0.0f || Rem.z != 0.0f) {
                    const long long o = out_index(S, pid);
                    atomicAdd(out + 3 * o + 0, Rem.x * scale);
                    atomicAdd(out + 3 * o + 1, Rem.y * scale);
                    atomicAdd(out + 3 * o + 2, Rem.z * scale);
                }
                alive = false;
            }
        }
        {
            const unsigned long long slot = reserve_slots(wv.count, njobs);
            if (njobs) {
                put_job(wv.jobs, slot, jx, jd, jw, job_key(pid, jfork));
                if (njobs == 2) put_job(wv.jobs, slot + 1, jx, M.sun_dir, jw2, job_key(pid, jfork + 1));
            }
        }
    }
    flush_counters(sc, n_paths_done, n_verts, tl);
}

template <int TR>
__global__ void __launch_bounds__(256, 4) k_shadow_fw(DMedium M, PathSrc S, const ShadowJob* __restrict__ jobs,
                                                   const unsigned long long* __restrict__ count, uint64_t seed,
                                                   float* out, float scale, DScratch* sc) {
    const unsigned long long n = *count;
    Tally tl;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const float4* p = reinterpret_cast<const float4*>(jobs + i);
        const float4 a = __ldcs(p), b = __ldcs(p + 1), c = __ldcs(p + 2);
        const float3 x = make_float3(a.x, a.y, a.z), dir = make_float3(a.w, b.x, b.y);
        const float3 wt = make_float3(b.z, b.w, c.x);
        const unsigned long long key = (unsigned long long)__float_as_uint(c.z) |
                                       ((unsigned long long)__float_as_uint(c.w) << 32);
        const uint64_t pid = key >> 16;
        Rng r;
        r.init(seed, pid, 2u * (1u + (uint32_t)(key & 0xffffu)));  // fork j of the path's stream 0
        float T;
        if (TR == 0) T = transmittance_rt(M, r, x, dir, tl, &sc->status);
        else if (TR == 1) T = transmittance_dt(M, r, x, dir, tl, &sc->status);
        else if (TR == 2) T = transmittance_dda<false>(M, x, dir, tl);
        else T = transmittance_dda<true>(M, x, dir, tl);
        const float3 c3 = wt * T;
        if (c3.x != 0.0f || c3.y != 0.0f || c3.z != 0.0f) {
            const long long o = out_index(S, pid);
            atomicAdd(out + 3 * o + 0, c3.x * scale);
            atomicAdd(out + 3 * o + 1, c3.y * scale);
            atomicAdd(out + 3 * o + 2, c3.z * scale);
        }
    }
    flush_counters(sc, 0, 0, tl);
}

// Host: rounds of walk + shadow until every path has been taken.
int launch_wave_fw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                   float scale, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.max_bounces <= 0) return VRT_E_UNSUPPORTED;
    const int lights = M.has_sun ? 2 : 1;
    const unsigned long long per_path = 1ull + (unsigned long long)lights * (unsigned long long)M.max_bounces;
    int blocks = persistent_blocks((const void*)k_walk_fw, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)need;
    const unsigned long long reserve = (unsigned long long)blocks * 256ull * per_path;
    unsigned long long cap = 3ull * reserve;
    if (cap < (1ull << 24)) cap = 1ull << 24;
    int st = ensure_wave_buffer(ctx, 256 + cap * sizeof(ShadowJob));
    if (st) {  // fall back to a smaller buffer (still > reserve)
        cap = reserve + reserve / 2;
        if ((st = ensure_wave_buffer(ctx, 256 + cap * sizeof(ShadowJob)))) return st;
    }
    WaveFw wv;
    wv.count = reinterpret_cast<unsigned long long*>(ctx->wave);
    wv.jobs = reinterpret_cast<ShadowJob*>(static_cast<char*>(ctx->wave) + 256);
    wv.cap = cap;
    wv.reserve = reserve;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const int sblocks = ctx->num_sms * 8;
    for (int round = 0;; ++round) {
        if ((e = cudaMemsetAsync(wv.count, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        k_walk_fw<<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, ctx->scratch, wv);
        switch (M.tr_mode) {
            case 0: k_shadow_fw<0><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
            case 1: k_shadow_fw<1><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
            case 2: k_shadow_fw<2><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
            default: k_shadow_fw<3><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
        }
        count_launches(2);
        if ((st = launch_status(cudaGetLastError()))) return st;
        unsigned long long taken = 0;
        if ((e = cudaMemcpyAsync(&taken, &ctx->scratch->next_path, sizeof(taken), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return launch_status(e);
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
        if (taken >= n_paths) break;
        if (round > (1 << 20)) return VRT_E_ITER_CAP;
    }
    return 0;
}

}  // namespace vrt
