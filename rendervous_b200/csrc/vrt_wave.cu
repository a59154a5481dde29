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
                                        unsigned long long key, uint32_t tgt = 0u) {
    float4* p = reinterpret_cast<float4*>(J + slot);
    p[0] = make_float4(x.x, x.y, x.z, d.x);
    p[1] = make_float4(d.y, d.z, wt.x, wt.y);
    p[2] = make_float4(wt.z, __uint_as_float(tgt), __uint_as_float((uint32_t)key), __uint_as_float((uint32_t)(key >> 32)));
}

struct JobView {
    float3 x, dir, wt;
    uint64_t pid;
    uint32_t fork, tgt;
};
__device__ __forceinline__ JobView get_job(const ShadowJob* J, unsigned long long i) {
    const float4* p = reinterpret_cast<const float4*>(J + i);
    const float4 a = __ldcs(p), b = __ldcs(p + 1), c = __ldcs(p + 2);
    JobView v;
    v.x = make_float3(a.x, a.y, a.z);
    v.dir = make_float3(a.w, b.x, b.y);
    v.wt = make_float3(b.z, b.w, c.x);
    v.tgt = __float_as_uint(c.y);
    const unsigned long long key = (unsigned long long)__float_as_uint(c.z) | ((unsigned long long)__float_as_uint(c.w) << 32);
    v.pid = key >> 16;
    v.fork = (uint32_t)(key & 0xffffu);
    return v;
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

// Per-warp sums of the lanes' tallies into the context counters.  `verts`
// counts forward path vertices only (the metric's unit); adjoint kernels pass 0.
__device__ __forceinline__ void flush_counters(DScratch* sc, uint32_t paths, uint32_t verts, const Tally& tl) {
    unsigned long long p = paths, v = verts, s = tl.steps, l = tl.lookups, a = tl.albedo, r = tl.reds;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(kAll, p, o);
        v += __shfl_down_sync(kAll, v, o);
        s += __shfl_down_sync(kAll, s, o);
        l += __shfl_down_sync(kAll, l, o);
        a += __shfl_down_sync(kAll, a, o);
        r += __shfl_down_sync(kAll, r, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (p) atomicAdd(&sc->paths, p);
        if (v) atomicAdd(&sc->vertices, v);
        if (s) atomicAdd(&sc->steps, s);
        if (l) atomicAdd(&sc->lookups, l);
        if (a) atomicAdd(&sc->albedo, a);
        if (r) atomicAdd(&sc->reds, r);
    }
}

// a device guard fired: the error code plus the site (VRT_E_ITER_CAP in both)
__device__ __forceinline__ void guard(DScratch* sc, int site) {
    atomicOr(&sc->status, 1u << 4);
    atomicOr(&sc->detail, 1u << site);
}

__device__ __forceinline__ long long out_index(const PathSrc& S, uint64_t pid) {
    return S.is_camera ? (long long)(pid % (uint64_t)S.npix) : (long long)pid;
}

template <int TR>
__device__ __forceinline__ float shadow_T(const DMedium& M, Rng& r, float3 x, float3 dir, Tally& tl, uint32_t* status) {
    if (TR == 0) return transmittance_rt(M, r, x, dir, tl, status);
    if (TR == 1) return transmittance_dt(M, r, x, dir, tl, status);
    if (TR == 2) return transmittance_dda<false>(M, x, dir, tl);
    return transmittance_dda<true>(M, x, dir, tl);
}

// The primary ray of path pid (camera or ray input), with the camera's draws.
__device__ __forceinline__ void start_ray(const PathSrc& S, uint64_t pid, Rng& rng, float3& x0, float3& w0) {
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
}

// Jobs a round aims to hold beyond the reserve: twice the expected count of
// the launch (two per path and light), at least 2^20 and at most 2^25.
inline unsigned long long batch_jobs(uint64_t n_paths, unsigned long long per_path) {
    unsigned long long c = (unsigned long long)n_paths * per_path * 2ull;
    if (c < (1ull << 20)) c = 1ull << 20;
    if (c > (1ull << 25)) c = 1ull << 25;
    return c;
}

// ---------------------------------------------------------------------------
// A shadow ray advanced one event per call: a majorant-brick crossing or a
// tracking collision.  The draws and arithmetic are those of transmittance_rt
// / transmittance_dt (vr_transmittance_RT.h:1-49, _DT.h:1-28) and of the first
// pass of their adjoints (_RT.h:51-98, _DT.h:30-62, majorant + 0.1); kernels
// that run one event per loop iteration for every lane keep the warp in one
// code path while rays of different lengths finish and are replaced.
// ---------------------------------------------------------------------------
struct ShadowRay {
    float3 x, dir;
    float d, T;
    Flight ff;
    Rng r;
    int it;
};

// Starts the ray (x, dir) on fork `fork` of path pid; false when it misses the
// medium (T = 1).
__device__ __forceinline__ bool shadow_begin(const DMedium& M, ShadowRay& s, float3 x, float3 dir, uint64_t seed,
                                             uint64_t pid, uint32_t fork) {
    s.r.init(seed, pid, 2u * (1u + fork));
    s.T = 1.0f;
    s.it = 0;
    s.ff = Flight();
    s.dir = dir;
    float tMin, tMax;
    if (!boundary(M, x, dir, tMin, tMax)) return false;
    s.x = x + dir * tMin;
    s.d = tMax - tMin;
    return true;
}

// One step: brick crossings (at most kCross) up to the next tracking
// collision, then that collision.  TR 0 ratio tracking, 1 delta tracking; BW:
// the adjoint's first pass (majorant + 0.1, ratio-tracking roulette below
// 0.1).  The lanes of a warp cross bricks in the inner loop and meet for the
// expensive part (sigma gather, draws), which thus runs with most lanes
// active.  Returns true when the estimate is complete (s.T).  On a tracking
// collision that continues the ray, hit is set with the majorant and the
// factor the adjoint's second pass scatters with (RT: r = 1 - sigma/maj; DT:
// Pc = sigma/maj).
constexpr int kCross = 16;

template <int TR, bool BW>
__device__ __forceinline__ bool shadow_event(const DMedium& M, ShadowRay& s, Tally& tl, DScratch* sc, bool& hit,
                                             float& hmaj, float& hf) {
    hit = false;
    const float EPS = 0.0000001f;
    float md, maj, t;
    for (int c = 0;; ++c) {
        if (++s.it > kStepCap) {
            raise_status(&sc->status, 4);
            return true;
        }
        const float q = s.ff.bk.query(M, s.x, s.dir, md);
        maj = BW ? gmax(EPS, q + 0.1f) : gmax(EPS, q);
        if (!BW && s.ff.tau < 0.0f) ++tl.steps;
        if (TR == 0) {
            t = s.ff.sample(s.r) / maj;
            if (md < s.d && t > md) {
                s.x = s.x + s.dir * md;
                s.d -= md;
                s.ff.cross(maj, md);
                s.ff.bk.advance(M);
                if (c + 1 >= kCross) return false;
                continue;
            }
        } else {
            const float dt = s.ff.sample(s.r) / maj;
            t = gmin(md, dt);
            s.x = s.x + s.dir * t;
            s.d -= t;
            if (s.d <= EPS) {
                s.T = 1.0f;
                return true;
            }
            if (dt > md) {
                s.ff.cross(maj, md);
                s.ff.bk.advance(M);
                if (c + 1 >= kCross) return false;
                continue;
            }
        }
        break;
    }
    if (TR == 0) {
        s.ff.used();
        const float dt = gmin(t, gmin(s.d, md));
        s.ff.bk.move(dt);
        s.x = s.x + s.dir * dt;
        s.d -= dt;
        if (s.d <= EPS) return true;
        const float r = 1.0f - sigma(M, s.x, tl) / maj;
        s.T *= r;
        if (s.T < (BW ? 0.1f : 0.01f)) {
            if (s.r.uniform() < 1.0f - s.T) {
                s.T = 0.0f;
                return true;
            }
            s.T = 1.0f;
        }
        hit = true;
        hmaj = maj;
        hf = r;
        return false;
    } else {
        s.ff.used();
        s.ff.bk.move(t);
        const float Pc = sigma(M, s.x, tl) / maj;
        if (s.r.uniform() < Pc) {
            s.T = 0.0f;
            return true;
        }
        hit = true;
        hmaj = maj;
        hf = Pc;
        return false;
    }
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
                    guard(sc, 0);
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
                guard(sc, 1);
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
        const JobView jv = get_job(jobs, i);
        Rng r;
        r.init(seed, jv.pid, 2u * (1u + jv.fork));  // fork j of the path's stream 0
        const float T = shadow_T<TR>(M, r, jv.x, jv.dir, tl, &sc->status);
        const float3 c3 = jv.wt * T;
        if (c3.x != 0.0f || c3.y != 0.0f || c3.z != 0.0f) {
            const long long o = out_index(S, jv.pid);
            atomicAdd(out + 3 * o + 0, c3.x * scale);
            atomicAdd(out + 3 * o + 1, c3.y * scale);
            atomicAdd(out + 3 * o + 2, c3.z * scale);
        }
    }
    flush_counters(sc, 0, 0, tl);
}

namespace {
constexpr uint32_t kNone = 0xffffffffu;
// A primal vertex of the NEE_DS adjoint wavefront: its two shadow
// transmittances and the next vertex of the same path.
struct VertexRec {
    float Te, Ts;
    uint32_t next, pad;
};
}  // namespace

// ---------------------------------------------------------------------------
// Persistent shadow kernels for ratio / delta tracking: one event per lane per
// iteration, finished lanes refilled from the job buffer with one atomic per
// warp (ranks from a ballot).
// ---------------------------------------------------------------------------
struct ShadowOut {
    float* out;        // OUT_IMAGE: image / ray radiance
    float scale;
    VertexRec* recs;   // OUT_RECORD: vertex records and per-path R / Rsp
    float* info;
    uint64_t p_begin;
};
enum : int { OUT_IMAGE = 0, OUT_RECORD = 1 };

template <int OUT>
__device__ __forceinline__ void shadow_finish(const PathSrc& S, const ShadowOut& so, const JobView& jv, float T) {
    if (OUT == OUT_RECORD) {
        VertexRec* rp = so.recs + (jv.tgt >> 2);
        if (jv.tgt & 1u) rp->Ts = T;
        else rp->Te = T;
    }
    const float3 c3 = jv.wt * T;
    if (c3.x != 0.0f || c3.y != 0.0f || c3.z != 0.0f) {
        if (OUT == OUT_IMAGE) {
            float* o = so.out + 3 * out_index(S, jv.pid);
            atomicAdd(o + 0, c3.x * so.scale);
            atomicAdd(o + 1, c3.y * so.scale);
            atomicAdd(o + 2, c3.z * so.scale);
        } else {
            float* o = so.info + 8 * (jv.pid - so.p_begin) + ((jv.tgt & 2u) ? 3 : 0);
            atomicAdd(o + 0, c3.x);
            atomicAdd(o + 1, c3.y);
            atomicAdd(o + 2, c3.z);
        }
    }
}

template <int TR, int OUT>
__global__ void __launch_bounds__(256, 4) k_shadow_run(DMedium M, PathSrc S, const ShadowJob* __restrict__ jobs,
                                                     const unsigned long long* __restrict__ count,
                                                     unsigned long long cap, unsigned long long* head, uint64_t seed,
                                                     ShadowOut so, DScratch* sc) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long n = *count;
    if (n > cap) n = cap;
    ShadowRay s;
    JobView jv;
    bool alive = false, exhausted = false;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(head, (unsigned long long)__popc(want));
            base = __shfl_sync(kAll, base, leader);
            if (!alive && !exhausted) {
                const unsigned long long i = base + __popc(want & ((1u << lane) - 1u));
                if (i >= n) {
                    exhausted = true;
                } else {
                    jv = get_job(jobs, i);
                    alive = shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork);
                    if (!alive) shadow_finish<OUT>(S, so, jv, 1.0f);
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;
        if (alive) {
            bool hit;
            float hm, hf;
            if (shadow_event<TR, false>(M, s, tl, sc, hit, hm, hf)) {
                shadow_finish<OUT>(S, so, jv, s.T);
                alive = false;
            }
        }
    }
    flush_counters(sc, 0, 0, tl);
}

// The transmittance adjoint (vr_transmittance_RT.h:51-141 / _DT.h:30-90): the
// first pass runs as events and keeps its tracking collisions; the second pass
// of the reference replays the same draws and scatters at exactly those
// points, so the scatter is done from the kept list once the first pass's
// estimate is known.  A ray with more than kKeep collisions replays its
// second pass as events instead.
constexpr int kKeep = 16;

template <int TR>
__global__ void __launch_bounds__(256, 3) k_shadow_adj(DMedium M, const ShadowJob* __restrict__ jobs,
                                                     const unsigned long long* __restrict__ count,
                                                     unsigned long long cap, unsigned long long* head, uint64_t seed,
                                                     DScratch* sc) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned long long n = *count;
    if (n > cap) n = cap;
    ShadowRay s;
    JobView jv;
    float4 keep[kKeep];  // position, majorant
    float keepf[kKeep];  // RT: r; DT: Pc
    int nkeep = 0, phase = 0;  // 0 idle, 1 first pass, 2 second pass (more than kKeep collisions)
    float outT = 0.0f;
    bool exhausted = false;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kAll, phase == 0 && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(head, (unsigned long long)__popc(want));
            base = __shfl_sync(kAll, base, leader);
            if (phase == 0 && !exhausted) {
                const unsigned long long i = base + __popc(want & ((1u << lane) - 1u));
                if (i >= n) {
                    exhausted = true;
                } else {
                    jv = get_job(jobs, i);
                    nkeep = 0;
                    if (jv.wt.x != 0.0f && shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork)) phase = 1;
                }
            }
        }
        if (__all_sync(kAll, phase == 0 && exhausted)) break;
        if (phase != 0) {
            bool hit;
            float hm, hf;
            const bool done = shadow_event<TR, true>(M, s, tl, sc, hit, hm, hf);
            const float dLdT = jv.wt.x;
            if (phase == 1) {
                if (hit) {
                    if (nkeep < kKeep) {
                        keep[nkeep] = make_float4(s.x.x, s.x.y, s.x.z, hm);
                        keepf[nkeep] = hf;
                    }
                    ++nkeep;
                }
                if (done) {
                    outT = s.T;
                    if (outT == 0.0f || s.it > kStepCap) {
                        phase = 0;  // ended by the roulette, a collision or the step cap: no gradient
                    } else if (nkeep <= kKeep) {
                        for (int k = 0; k < nkeep; ++k) {
                            const float3 px = make_float3(keep[k].x, keep[k].y, keep[k].z);
                            const float g = TR == 0 ? -outT * dLdT / keep[k].w / keepf[k]
                                                    : -dLdT / keep[k].w / (1.0f - keepf[k]);
                            sigma_bw(M, px, g, tl);
                        }
                        phase = 0;
                    } else {  // replay the second pass
                        shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork);
                        phase = 2;
                    }
                }
            } else {
                if (hit) {
                    const float g = TR == 0 ? -outT * dLdT / hm / hf : -dLdT / hm / (1.0f - hf);
                    sigma_bw(M, s.x, g, tl);
                }
                if (done) phase = 0;
            }
        }
    }
    flush_counters(sc, 0, 0, tl);
}

// Host: rounds of walk + shadow until every path has been taken.
int launch_wave_fw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                   float scale, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.max_bounces <= 0) return VRT_E_UNSUPPORTED;
    const unsigned long long lights = M.has_sun ? 2ull : 1ull;
    const unsigned long long per_path = 1ull + lights * (unsigned long long)M.max_bounces;
    int blocks = persistent_blocks((const void*)k_walk_fw, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)need;
    // the worst case of every path in flight, plus room for a round's expected jobs
    unsigned long long inflight = (unsigned long long)blocks * 256ull;
    if (inflight > n_paths) inflight = n_paths;
    const unsigned long long reserve = inflight * per_path;
    const unsigned long long cap = reserve + batch_jobs(n_paths, 1ull + lights);
    int st = ensure_wave_buffer(ctx, 256 + cap * sizeof(ShadowJob));
    if (st) return st;
    WaveFw wv;
    wv.count = reinterpret_cast<unsigned long long*>(ctx->wave);
    wv.jobs = reinterpret_cast<ShadowJob*>(static_cast<char*>(ctx->wave) + 256);
    wv.cap = cap;
    wv.reserve = reserve;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const int sblocks = ctx->num_sms * 8;
    const int rblocks = persistent_blocks(M.tr_mode == 0 ? (const void*)k_shadow_run<0, OUT_IMAGE>
                                                         : (const void*)k_shadow_run<1, OUT_IMAGE>, 256, ctx->num_sms);
    const ShadowOut so = {out, scale, nullptr, nullptr, 0};
    for (int round = 0;; ++round) {
        // count of the jobs written, and the head the persistent shadow kernel takes them from
        if ((e = cudaMemsetAsync(wv.count, 0, 2 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        k_walk_fw<<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, ctx->scratch, wv);
        switch (M.tr_mode) {
            case 0: k_shadow_run<0, OUT_IMAGE><<<rblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, wv.cap, wv.count + 1, seed, so, ctx->scratch); break;
            case 1: k_shadow_run<1, OUT_IMAGE><<<rblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, wv.cap, wv.count + 1, seed, so, ctx->scratch); break;
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

// ------------------------------------------------------------------------
// NEE_DS adjoint (include/vr_path_integrator_NEE_DS.h:6-206) as a wavefront.
//
// With the default replay majorant (the primal's) the replay retraces the
// primal's vertices exactly -- same draws, same throughputs, and shadow j of
// the path draws from fork j in both passes -- so a vertex's shadow
// transmittances are computed once and stored, and the transmittance adjoints
// (which feed nothing back into the path) run as independent jobs:
//
//   A k_ds_primal   the primal walk: per real collision a vertex record (linked
//                   per path) and a T job per light; per path the emission and
//                   escape terms of R and Rsp
//   B k_shadow_T    T of each job into its record, weight * T into its path's
//                   R (or Rsp after a zero-density collision)
//   C k_ds_replay   the replay walk: dL/dsigma at every collision, dL/dalbedo
//                   at real ones, the R bookkeeping from the stored T, and a
//                   transmittance-adjoint job per light with dL/dT != 0
//   D k_shadow_bw   the two-pass ratio / delta tracking adjoint or the DDA
//                   adjoint of each job
//
// Rounds bound the buffers as in the forward wavefront.
// ------------------------------------------------------------------------

struct WaveBw {
    ShadowJob* jobs;
    VertexRec* recs;
    float* info;               // per path: R (3), Rsp (3), first record, pad
    unsigned long long* hdr;   // [0] jobs, [1] records, [2] replay queue
    unsigned long long cap_jobs, cap_recs, cap_paths;
    unsigned long long res_jobs, res_recs, lanes;
    uint64_t p_begin;
};

__global__ void __launch_bounds__(256, 4) k_ds_primal(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                    DScratch* sc, WaveBw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    const int lights = M.has_sun ? 2 : 1;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f), Racc = f3(0.0f), Rspacc = f3(0.0f);
    float d = 0.0f, null_W = 1.0f;
    bool scattered = false, alive = false, exhausted = false;
    int bounces = 0;
    uint64_t pid = 0;
    uint32_t steps_path = 0, first = kNone, prev = kNone;
    uint32_t n_paths_done = 0;
    Tally tl;

    while (true) {
        unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) {
                const unsigned long long uj = *((volatile unsigned long long*)&wv.hdr[0]);
                const unsigned long long ur = *((volatile unsigned long long*)&wv.hdr[1]);
                const unsigned long long up = *((volatile unsigned long long*)&sc->next_path) - wv.p_begin;
                const bool room = uj + wv.res_jobs <= wv.cap_jobs && ur + wv.res_recs <= wv.cap_recs &&
                                  up + wv.lanes <= wv.cap_paths;
                base = room ? atomicAdd(&sc->next_path, (unsigned long long)__popc(want)) : ~0ull;
            }
            base = __shfl_sync(kAll, base, leader);
            if (base == ~0ull) {
                exhausted = true;
            } else if (!alive && !exhausted) {
                const uint64_t p = base + __popc(want & ((1u << lane) - 1u));
                if (p >= n_paths) {
                    exhausted = true;
                } else {
                    pid = p;
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    start_ray(S, pid, rng, x0, w0);
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    x = x0 + w0 * tMin;
                    w = w0;
                    d = tMax - tMin;
                    W = f3(1.0f);
                    Racc = f3(0.0f);
                    Rspacc = f3(0.0f);
                    null_W = 1.0f;
                    scattered = false;
                    bounces = 0;
                    steps_path = 0;
                    first = kNone;
                    prev = kNone;
                    ff = Flight();
                    alive = true;
                    ++n_paths_done;
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        int nrec = 0, nj = 0;
        bool finish = false, rsp = false;
        float3 wnee = f3(0.0f), we = f3(0.0f), ws = f3(0.0f);
        uint32_t jfork = 0;
        if (alive) {
            int ev = 0;  // 0 none, 1 collision, 2 end
            if (!(d > EPS)) {
                ev = 2;  // the while (d > EPS) test (_NEE_DS.h:31)
            } else {
                bool need = false;
                float m = 0.0f, t = 0.0f;
                if (ff.tau < 0.0f) ++tl.steps;
                ff.sample(rng);
                for (int k = 0;; ++k) {
                    if (k >= kStepCap) {
                        guard(sc, 2);
                        ev = 2;
                        break;
                    }
                    float md;
                    m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps + 0.1f);  // _NEE_DS.h:36
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
                    else need = true;
                    ff.bk.move(t);
                    break;
                }
                if (need) {
                    const float s = sigma(M, x, tl);
                    const float Pc = (s + eps) / m;
                    if (rng.uniform() >= Pc) {  // null collision (_NEE_DS.h:41-45)
                        W = W * ((1.0f - s / m) / (1.0f - Pc));
                        d -= t;
                    } else {  // real collision (_NEE_DS.h:48-99)
                        scattered = true;
                        bool dead = false;
                        if (s < EPS) {
                            if (null_W < EPS) { W = f3(0.0f); dead = true; }
                            else null_W = 0.0f;
                        } else {
                            W = W * ((s / m) / Pc);
                        }
                        if (dead) {
                            ev = 2;
                        } else {
                            const float3 sa = albedo(M, x, tl);
                            const float3 acc = W * (f3(1.0f) - sa) * M.emission;
                            W = W * sa;
                            const float3 Le = environment_sample(M, rng, wnee);
                            we = W * Le * phase(M, w, wnee);
                            if (M.has_sun) ws = W * M.sun_L * phase(M, w, M.sun_dir);
                            jfork = rng.ntr;
                            rng.ntr += (uint32_t)lights;
                            const bool capped = M.max_bounces > 0 && bounces + 1 >= M.max_bounces;
                            float3 wo = w;
                            if (!capped) wo = phase_sample(M, rng, w);
                            rsp = null_W < EPS;
                            if (rsp) Rspacc = Rspacc + acc;
                            else Racc = Racc + acc;
                            nrec = 1;
                            nj = lights;
                            ++bounces;
                            if (capped || all_less(W, EPS)) {
                                W = f3(0.0f);
                                ev = 2;
                            } else {
                                w = wo;
                                float tMin;
                                boundary(M, x, w, tMin, d);
                                ff = Flight();
                            }
                        }
                    }
                }
            }
            if (++steps_path > (uint32_t)kPathCap) {
                guard(sc, 3);
                ev = 2;
            }
            finish = ev == 2;
        }
        // ---- the vertex record (linked to the path's previous one) and its T jobs
        const unsigned long long r = reserve_slots(&wv.hdr[1], nrec);
        if (nrec) {
            VertexRec* rp = wv.recs + r;
            rp->Te = 1.0f;
            rp->Ts = 1.0f;
            rp->next = kNone;
            if (first == kNone) first = (uint32_t)r;
            else wv.recs[prev].next = (uint32_t)r;
            prev = (uint32_t)r;
        }
        const unsigned long long j = reserve_slots(&wv.hdr[0], nj);
        if (nj) {
            const uint32_t tgt = ((uint32_t)r << 2) | (rsp ? 2u : 0u);
            put_job(wv.jobs, j, x, wnee, we, job_key(pid, jfork), tgt);
            if (nj == 2) put_job(wv.jobs, j + 1, x, M.sun_dir, ws, job_key(pid, jfork + 1), tgt | 1u);
        }
        if (finish) {  // end of the primal (_NEE_DS.h:106-110): escape term, then the path's totals
            if (!scattered) Racc = Racc + M.env * W;
            float* io = wv.info + 8 * (pid - wv.p_begin);
            reinterpret_cast<float4*>(io)[0] = make_float4(Racc.x, Racc.y, Racc.z, Rspacc.x);
            reinterpret_cast<float4*>(io)[1] = make_float4(Rspacc.y, Rspacc.z, __uint_as_float(first), 0.0f);
            alive = false;
        }
    }
    flush_counters(sc, n_paths_done, 0, tl);  // the forward counts the vertices
}

template <int TR>
__global__ void __launch_bounds__(256, 4) k_shadow_T(DMedium M, WaveBw wv, uint64_t seed, DScratch* sc) {
    const unsigned long long n = wv.hdr[0];
    Tally tl;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const JobView jv = get_job(wv.jobs, i);
        Rng r;
        r.init(seed, jv.pid, 2u * (1u + jv.fork));
        const float T = shadow_T<TR>(M, r, jv.x, jv.dir, tl, &sc->status);
        VertexRec* rp = wv.recs + (jv.tgt >> 2);
        if (jv.tgt & 1u) rp->Ts = T;
        else rp->Te = T;
        const float3 c3 = jv.wt * T;
        if (c3.x != 0.0f || c3.y != 0.0f || c3.z != 0.0f) {
            float* io = wv.info + 8 * (jv.pid - wv.p_begin) + ((jv.tgt & 2u) ? 3 : 0);
            atomicAdd(io + 0, c3.x);
            atomicAdd(io + 1, c3.y);
            atomicAdd(io + 2, c3.z);
        }
    }
    flush_counters(sc, 0, 0, tl);
}

__global__ void __launch_bounds__(256, 3) k_ds_replay(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                    const float* __restrict__ dL, float div, DScratch* sc, WaveBw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    const int lights = M.has_sun ? 2 : 1;
    unsigned long long p_end = *((volatile unsigned long long*)&sc->next_path);
    if (p_end > n_paths) p_end = n_paths;
    const unsigned long long n_round = p_end - wv.p_begin;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f), R = f3(0.0f), Rsp = f3(0.0f), dLdR = f3(0.0f);
    float d = 0.0f;
    bool alive = false, exhausted = false;
    int bounces = 0;
    uint64_t pid = 0;
    uint32_t steps_path = 0, cur = kNone;
    Tally tl;

    while (true) {
        unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&wv.hdr[2], (unsigned long long)__popc(want));
            base = __shfl_sync(kAll, base, leader);
            if (!alive && !exhausted) {
                const unsigned long long k = base + __popc(want & ((1u << lane) - 1u));
                if (k >= n_round) {
                    exhausted = true;
                } else {
                    pid = wv.p_begin + k;
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    start_ray(S, pid, rng, x0, w0);
                    dLdR = ld3(dL + 3 * out_index(S, pid)) / div;
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    x = x0 + w0 * tMin;
                    w = w0;
                    d = tMax - tMin;
                    W = f3(1.0f);
                    bounces = 0;
                    steps_path = 0;
                    const float4* io = reinterpret_cast<const float4*>(wv.info + 8 * k);
                    const float4 a = io[0], b = io[1];
                    R = make_float3(a.x, a.y, a.z);
                    Rsp = make_float3(a.w, b.x, b.y);
                    cur = __float_as_uint(b.z);
                    ff = Flight();
                    alive = true;
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        int nj = 0;
        float3 jd0 = f3(0.0f), jd1 = f3(0.0f);
        float dT0 = 0.0f, dT1 = 0.0f;
        uint32_t f0 = 0, f1 = 0;
        if (alive) {
            int ev = 0;
            if (!(d > EPS)) {
                ev = 2;
            } else {
                bool need = false;
                float m = 0.0f, t = 0.0f;
                if (ff.tau < 0.0f) ++tl.steps;
                ff.sample(rng);
                for (int k = 0;; ++k) {
                    if (k >= kStepCap) {
                        guard(sc, 4);
                        ev = 2;
                        break;
                    }
                    float md;
                    m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps + 0.1f);
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
                    else need = true;
                    ff.bk.move(t);
                    break;
                }
                if (need) {
                    const float s = sigma(M, x, tl);
                    const float Pc = (s + eps) / m;
                    float gsc;
                    const bool real = !(rng.uniform() >= Pc);
                    if (!real) {  // _NEE_DS.h:130-140
                        gsc = dot(dLdR, -R / m / (1.0f - s / m));
                        W = W * ((1.0f - s / m) / (1.0f - Pc));
                        d -= t;
                    } else {      // _NEE_DS.h:142-150
                        gsc = dot(dLdR, s < EPS ? Rsp / eps : R / s);
                    }
                    if (gsc != 0.0f) sigma_bw(M, x, gsc, tl);
                    if (real) {   // replayed vertex (_NEE_DS.h:151-203)
                        W = W * (s / m / Pc);
                        if (s < EPS) {
                            ev = 2;
                        } else {
                            const float3 sa = albedo(M, x, tl);
                            float3 dL_dsa = dLdR * W * -1.0f * M.emission;
                            R = R - W * (f3(1.0f) - sa) * M.emission;
                            dL_dsa = dL_dsa + dLdR * R / make_float3(gmax(EPS, sa.x), gmax(EPS, sa.y), gmax(EPS, sa.z));
                            albedo_bw(M, x, dL_dsa, tl);
                            float3 wnee;
                            const float3 Le = environment_sample(M, rng, wnee);
                            const float ph_nee = phase(M, w, wnee);
                            const float ph_sun = M.has_sun ? phase(M, w, M.sun_dir) : 0.0f;
                            const uint32_t jf = rng.ntr;
                            rng.ntr += (uint32_t)lights;
                            const float3 wo = phase_sample(M, rng, w);
                            W = W * sa;
                            float Te = 1.0f, Ts = 1.0f;
                            if (cur == kNone) {
                                guard(sc, 5);  // the replay left the primal's path
                                ev = 2;
                            } else {
                                const VertexRec rec = wv.recs[cur];
                                Te = rec.Te;
                                Ts = rec.Ts;
                                cur = rec.next;
                            }
                            if (ev != 2) {
                                const float dTe = dot(dLdR, W * Le * ph_nee);
                                R = R - W * Te * Le * ph_nee;
                                if (dTe != 0.0f) { jd0 = wnee; dT0 = dTe; f0 = jf; nj = 1; }
                                if (M.has_sun) {
                                    const float dTs = dot(dLdR, W * M.sun_L * ph_sun);
                                    R = R - W * Ts * M.sun_L * ph_sun;
                                    if (dTs != 0.0f) {
                                        if (nj == 0) { jd0 = M.sun_dir; dT0 = dTs; f0 = jf + 1; nj = 1; }
                                        else { jd1 = M.sun_dir; dT1 = dTs; f1 = jf + 1; nj = 2; }
                                    }
                                }
                                ++bounces;
                                if ((M.max_bounces > 0 && bounces >= M.max_bounces) || all_less(W, EPS)) {
                                    ev = 2;
                                } else {
                                    w = wo;
                                    float tMin;
                                    boundary(M, x, w, tMin, d);
                                    ff = Flight();
                                }
                            }
                        }
                    }
                }
            }
            if (++steps_path > (uint32_t)kPathCap) {
                guard(sc, 6);
                ev = 2;
            }
            if (ev == 2) alive = false;
        }
        const unsigned long long j = reserve_slots(&wv.hdr[0], nj);
        if (nj) {
            if (j + (unsigned long long)nj > wv.cap_jobs) {
                guard(sc, 7);
            } else {
                put_job(wv.jobs, j, x, jd0, make_float3(dT0, 0.0f, 0.0f), job_key(pid, f0));
                if (nj == 2) put_job(wv.jobs, j + 1, x, jd1, make_float3(dT1, 0.0f, 0.0f), job_key(pid, f1));
            }
        }
    }
    flush_counters(sc, 0, 0, tl);
}

template <int TR>
__global__ void __launch_bounds__(256, 4) k_shadow_bw(DMedium M, WaveBw wv, uint64_t seed, DScratch* sc) {
    unsigned long long n = wv.hdr[0];
    if (n > wv.cap_jobs) n = wv.cap_jobs;
    Tally tl;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const JobView jv = get_job(wv.jobs, i);
        Rng r;
        r.init(seed, jv.pid, 2u * (1u + jv.fork));
        if (TR == 0) transmittance_rt_bw(M, r, jv.x, jv.dir, jv.wt.x, tl, &sc->status);
        else if (TR == 1) transmittance_dt_bw(M, r, jv.x, jv.dir, jv.wt.x, tl, &sc->status);
        else if (TR == 2) transmittance_dda_bw<false>(M, jv.x, jv.dir, jv.wt.x, tl);
        else transmittance_dda_bw<true>(M, jv.x, jv.dir, jv.wt.x, tl);
    }
    flush_counters(sc, 0, 0, tl);
}

int launch_wave_ds_bw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                      const float* dL, float div, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.max_bounces <= 0 || M.ds_compat) return VRT_E_UNSUPPORTED;
    const unsigned long long lights = M.has_sun ? 2ull : 1ull, B = (unsigned long long)M.max_bounces;
    int blocksA = persistent_blocks((const void*)k_ds_primal, 256, ctx->num_sms);
    int blocksC = persistent_blocks((const void*)k_ds_replay, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocksA > need) blocksA = (int)need;
    if ((uint64_t)blocksC > need) blocksC = (int)need;
    WaveBw wv;
    wv.lanes = (unsigned long long)blocksA * 256ull;
    const unsigned long long inflight = wv.lanes < n_paths ? wv.lanes : n_paths;
    wv.res_jobs = inflight * lights * B;
    wv.res_recs = inflight * B;
    wv.cap_jobs = wv.res_jobs + batch_jobs(n_paths, lights);
    wv.cap_recs = wv.res_recs + batch_jobs(n_paths, 1);
    if (wv.cap_recs > (1ull << 30)) return VRT_E_UNSUPPORTED;  // record indices are 30-bit in a job
    wv.cap_paths = (n_paths < (1ull << 24) ? n_paths : (1ull << 24)) + wv.lanes;
    const size_t bytes = 256 + wv.cap_jobs * sizeof(ShadowJob) + wv.cap_recs * sizeof(VertexRec) + wv.cap_paths * 32;
    int st = ensure_wave_buffer(ctx, bytes);
    if (st) return st;
    char* base = static_cast<char*>(ctx->wave);
    wv.hdr = reinterpret_cast<unsigned long long*>(base);
    wv.jobs = reinterpret_cast<ShadowJob*>(base + 256);
    wv.recs = reinterpret_cast<VertexRec*>(base + 256 + wv.cap_jobs * sizeof(ShadowJob));
    wv.info = reinterpret_cast<float*>(base + 256 + wv.cap_jobs * sizeof(ShadowJob) + wv.cap_recs * sizeof(VertexRec));
    wv.p_begin = 0;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const int sblocks = ctx->num_sms * 8;
    const int tblocks = persistent_blocks(M.tr_mode == 0 ? (const void*)k_shadow_run<0, OUT_RECORD>
                                                         : (const void*)k_shadow_run<1, OUT_RECORD>, 256, ctx->num_sms);
    const int ablocks = persistent_blocks(M.tr_mode == 0 ? (const void*)k_shadow_adj<0> : (const void*)k_shadow_adj<1>,
                                          256, ctx->num_sms);
    ShadowOut sor = {nullptr, 0.0f, wv.recs, wv.info, 0};
    for (int round = 0;; ++round) {
        // [0] jobs, [1] records, [2] replay queue, [3] / [4] heads of the shadow kernels
        if ((e = cudaMemsetAsync(wv.hdr, 0, 5 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        sor.p_begin = wv.p_begin;
        k_ds_primal<<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
        switch (M.tr_mode) {
            case 0: k_shadow_run<0, OUT_RECORD><<<tblocks, 256, 0, stream>>>(M, src, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[3], seed, sor, ctx->scratch); break;
            case 1: k_shadow_run<1, OUT_RECORD><<<tblocks, 256, 0, stream>>>(M, src, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[3], seed, sor, ctx->scratch); break;
            case 2: k_shadow_T<2><<<sblocks, 256, 0, stream>>>(M, wv, seed, ctx->scratch); break;
            default: k_shadow_T<3><<<sblocks, 256, 0, stream>>>(M, wv, seed, ctx->scratch); break;
        }
        if ((e = cudaMemsetAsync(wv.hdr, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        k_ds_replay<<<blocksC, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, ctx->scratch, wv);
        switch (M.tr_mode) {
            case 0: k_shadow_adj<0><<<ablocks, 256, 0, stream>>>(M, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[4], seed, ctx->scratch); break;
            case 1: k_shadow_adj<1><<<ablocks, 256, 0, stream>>>(M, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[4], seed, ctx->scratch); break;
            case 2: k_shadow_bw<2><<<sblocks, 256, 0, stream>>>(M, wv, seed, ctx->scratch); break;
            default: k_shadow_bw<3><<<sblocks, 256, 0, stream>>>(M, wv, seed, ctx->scratch); break;
        }
        count_launches(4);
        if ((st = launch_status(cudaGetLastError()))) return st;
        unsigned long long taken = 0;
        if ((e = cudaMemcpyAsync(&taken, &ctx->scratch->next_path, sizeof(taken), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return launch_status(e);
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
        if (taken >= n_paths) break;
        wv.p_begin = taken;
        if (round > (1 << 20)) return VRT_E_ITER_CAP;
    }
    return 0;
}

}  // namespace vrt
