// vrt_wave.cuh -- pieces shared by the wavefront kernels: the shadow-job
// buffer, warp-aggregated slot reservation, counter flushes, and a shadow ray
// advanced one step at a time (vrt_wave.cu: forward walk and every shadow
// kernel; vrt_wave_ds.cu: the NEE_DS primal walk and its collision-log replay).
#pragma once
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include "vrt_tracking.cuh"

namespace vrt {
namespace wave {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kPathCap = 1 << 26;  // free-flight steps of one path before VRT_E_ITER_CAP

// 48 bytes: position, direction, weight, key = pid << 16 | fork
struct ShadowJob {
    float4 a, b, c;
};

__device__ __forceinline__ void put_job(ShadowJob* J, unsigned long long slot, float3 x, float3 d, float3 wt,
                                        unsigned long long key, uint32_t tgt = 0u) {
    float4* p = reinterpret_cast<float4*>(J + slot);
    // streaming stores: jobs are read once, by the next kernel; keep them from
    // evicting the grids' lines in L2
    __stcs(p, make_float4(x.x, x.y, x.z, d.x));
    __stcs(p + 1, make_float4(d.y, d.z, wt.x, wt.y));
    __stcs(p + 2, make_float4(wt.z, __uint_as_float(tgt), __uint_as_float((uint32_t)key),
                              __uint_as_float((uint32_t)(key >> 32))));
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
    if (!__any_sync(kAll, n != 0)) return 0;  // most iterations emit nothing: skip the scan
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

// Warp-aggregated reservation on four counters at once: the lanes' counts are
// packed a byte apiece (each warp total stays below 256), one shuffle scan
// gives every lane its offsets, and lanes 31, 30, 29 and 28 add the totals to
// counters 0..3.  Returns each lane's first slot per counter.
struct Slots4 {
    unsigned long long s0, s1, s2, s3;
};
__device__ __forceinline__ Slots4 reserve_slots4(unsigned long long* c0, unsigned long long* c1,
                                                 unsigned long long* c2, unsigned long long* c3, uint32_t packed) {
    Slots4 out = {0ull, 0ull, 0ull, 0ull};
    if (!__any_sync(kAll, packed != 0u)) return out;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t incl = packed;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(kAll, incl, o);
        if ((int)lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(kAll, incl, 31);
    unsigned long long b = 0;
    const unsigned f = 31u - lane;
    if (f < 4u) {
        const uint32_t t = (total >> (8u * f)) & 0xffu;
        unsigned long long* c = f == 0u ? c0 : (f == 1u ? c1 : (f == 2u ? c2 : c3));
        if (t) b = atomicAdd(c, (unsigned long long)t);
    }
    const uint32_t excl = incl - packed;
    out.s0 = __shfl_sync(kAll, b, 31) + (excl & 0xffu);
    out.s1 = __shfl_sync(kAll, b, 30) + ((excl >> 8) & 0xffu);
    out.s2 = __shfl_sync(kAll, b, 29) + ((excl >> 16) & 0xffu);
    out.s3 = __shfl_sync(kAll, b, 28) + (excl >> 24);
    return out;
}

// Work items [0, n) claimed from a global counter a chunk per warp: one atomic
// per `chunk` items instead of one per refill.  All lanes call take()
// together with the ballot of the lanes that want an item; a lane gets one
// (returns true, item set) while the warp's chunk lasts.  Lanes left over wait
// for the next call, which claims a new chunk; `drained` turns true when a
// claim finds the counter past n.
struct WarpQueue {
    unsigned long long next = 0, end = 0;
    bool drained = false;
    __device__ __forceinline__ bool take(unsigned long long* head, unsigned long long n, unsigned long long chunk,
                                         unsigned want, unsigned long long& item) {
        const unsigned lane = threadIdx.x & 31u;
        if (next >= end && !drained) {
            unsigned long long b = 0;
            if (lane == 0u) b = atomicAdd(head, chunk);
            b = __shfl_sync(kAll, b, 0);
            if (b >= n) {
                drained = true;
            } else {
                next = b;
                end = b + chunk < n ? b + chunk : n;
            }
        }
        const unsigned long long avail = next < end ? end - next : 0ull;
        const unsigned rank = __popc(want & ((1u << lane) - 1u));
        const bool got = ((want >> lane) & 1u) != 0u && (unsigned long long)rank < avail;
        item = next + rank;
        const unsigned long long used = (unsigned long long)__popc(want);
        next += used < avail ? used : avail;
        return got;
    }
};

// Per-warp sums of the lanes' tallies into the context counters.  `verts`
// counts forward path vertices only (the metric's unit); adjoint kernels pass 0.
__device__ __forceinline__ void flush_counters(DScratch* sc, int kid, uint32_t paths, uint32_t verts, const Tally& tl) {
    unsigned long long p = paths, v = verts, s = tl.steps, l = tl.lookups, a = tl.albedo, r = tl.reds, b = tl.logb;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        b += __shfl_down_sync(kAll, b, o);
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
        if (s) atomicAdd(&sc->kstat[kid][0], s);
        if (l) atomicAdd(&sc->kstat[kid][1], l);
        if (r) atomicAdd(&sc->kstat[kid][2], r);
        if (a) atomicAdd(&sc->kstat[kid][3], a);
        if (b) atomicAdd(&sc->kstat[kid][4], b);
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
    if (TR == 3) return transmittance_dda<true>(M, x, dir, tl);
    if (TR == 4) return transmittance_grid_tracking<false>(M, r, x, dir, tl, status);
    return transmittance_grid_tracking<true>(M, r, x, dir, tl, status);
}

// The primary ray of path pid (camera or ray input), with the camera's draws.
__device__ __forceinline__ void start_ray(const PathSrc& S, uint64_t pid, Rng& rng, float3& x0, float3& w0,
                                          DScratch* sc) {
    if (S.is_camera) {
        camera_pixel_ray(S.cam, (long long)(pid % (uint64_t)S.npix), rng, x0, w0, &sc->status);
    } else {
        x0 = ld3(S.rays + 6 * pid);
        w0 = ld3(S.rays + 6 * pid + 3);
    }
}

// Items a round aims to hold beyond the reserve: twice `per_path` per path,
// at least 2^20 and at most 2^27 (a 512x512 x 64 spp capture then runs in one
// round: fewer kernel tails and host syncs, for about 18 GB of HBM).
inline unsigned long long batch_jobs(uint64_t n_paths, unsigned long long per_path, unsigned long long limit = 0) {
    unsigned long long c = (unsigned long long)n_paths * per_path * 2ull;
    if (c < (1ull << 20)) c = 1ull << 20;
    if (c > (1ull << 27)) c = 1ull << 27;
    if (limit && c > limit) c = limit;  // vrt_set_wave_batch_limit: a smaller footprint, more rounds
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
// sbase: the stream the forks come from (0: the path's stream; 1: the DRT
// adjoint's stream for the transmittance adjoints).
__device__ __forceinline__ bool shadow_begin(const DMedium& M, ShadowRay& s, float3 x, float3 dir, uint64_t seed,
                                             uint64_t pid, uint32_t fork, uint32_t sbase = 0u) {
    s.r.init(seed, pid, sbase + 2u * (1u + fork));
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

// One step: brick crossings (at most kCross, kCrossBw in the adjoint's first
// pass) up to the next tracking
// collision, then that collision.  TR 0 ratio tracking, 1 delta tracking; BW:
// the adjoint's first pass (majorant + 0.1, ratio-tracking roulette below
// 0.1).  The lanes of a warp cross bricks in the inner loop and meet for the
// expensive part (sigma gather, draws), which thus runs with most lanes
// active.  Returns true when the estimate is complete (s.T).  On a tracking
// collision that continues the ray, hit is set with the majorant and the
// factor the adjoint's second pass scatters with (RT: r = 1 - sigma/maj; DT:
// Pc = sigma/maj).
constexpr int kCross = 6;    // forward transmittances (k_shadow_run)
constexpr int kCrossBw = 8;  // the transmittance adjoint's first pass (k_shadow_adj)
// The same bound for the path walks (measured per kernel): a flight that needs
// more brick crossings leaves the crossing loop without an event and resumes
// in the next iteration, so the warp's long flights do not hold the others.
constexpr int kWalkCross = 12;  // k_walk_fw
constexpr int kDsCross = 8;     // k_ds_primal, k_ds_rewalk

// Vertices an uncapped path (max_bounces == 0, the reference's default) walks
// in one pass of a wavefront; a longer path continues in a later pass
// (forward) or is run whole by the state-machine adjoint (NEE_DS).
constexpr int kUncappedPass = 64;

template <int TR, bool BW>
__device__ __forceinline__ bool shadow_event(const DMedium& M, ShadowRay& s, Tally& tl, DScratch* sc, bool& hit,
                                             float& hmaj, float& hf) {
    hit = false;
    const float EPS = 0.0000001f;
    float md, maj, t;
    // a flight draws its optical depth once (crossings keep it positive)
    if (!BW && s.ff.tau < 0.0f) ++tl.steps;
    s.ff.sample(s.r);
    for (int c = 0;; ++c) {
        if (++s.it > kStepCap) {
            raise_status(&sc->status, 4);
            return true;
        }
        const float q = s.ff.bk.query(M, s.x, s.dir, md);
        maj = BW ? gmax(EPS, q + 0.1f) : gmax(EPS, q);
        // the flight crosses the brick face when its optical depth exceeds
        // majorant x distance to the face: tested without a division, and the
        // crossing leaves the depth positive
        if (TR == 0) {
            const float tau = s.ff.tau;
            if (md < s.d && tau > md * maj) {
                s.x = s.x + s.dir * md;
                s.d -= md;
                s.ff.cross(maj, md);
                s.ff.bk.advance(M);
                if (c + 1 >= (BW ? kCrossBw : kCross)) return false;
                continue;
            }
            t = tau / maj;
        } else {
            const float tau = s.ff.tau;
            const bool crosses = tau > md * maj;
            t = md;
            if (!crosses) t = gmin(md, tau / maj);
            s.x = s.x + s.dir * t;
            s.d -= t;
            if (s.d <= EPS) {
                s.T = 1.0f;
                return true;
            }
            if (crosses) {
                s.ff.cross(maj, md);
                s.ff.bk.advance(M);
                if (c + 1 >= (BW ? kCrossBw : kCross)) return false;
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


constexpr uint32_t kNone = 0xffffffffu;
constexpr uint32_t kUnlogged = 0xfffffffeu;  // a path whose collisions did not fit the log
constexpr uint32_t kSpilled = 0xfffffffdu;   // a path handed to the state-machine adjoint
// the record word of a light job that only has a transmittance adjoint (the
// DRT adjoint's primary ray toward the environment): no T, no record
constexpr uint32_t kAdjOnly = 0xffffffffu;
// A real-collision vertex of the NEE_DS primal (48 bytes): its two shadow
// transmittances (filled by the shadow kernel), the next vertex of the same
// path, the slot of its environment job (the sun job follows it), and what the
// replay needs to redo the vertex without walking to it: the albedo, the
// environment radiance and the two phase values.  The transmittance adjoint
// of the vertex reuses the primal's jobs (same ray, same Philox fork), so the
// replay only stores dL/dT per job slot.
struct VertexRec {
    float Te, Ts;
    uint32_t next, job;
    float sa[3], ph_env;
    float Le[3], ph_sun;
};
static_assert(sizeof(VertexRec) == 48, "vertex records are three 16-byte words");

// One tracking collision of the NEE_DS primal (32 bytes, two 16-byte words):
// position and sigma there; majorant, next collision of the path, the vertex
// record (real collisions that scatter) and bit 0 = real collision.
struct CollisionRec {
    float4 xs;   // x, y, z, sigma
    uint4 link;  // majorant bits, next, record, flags
};
static_assert(sizeof(CollisionRec) == 32, "collision records are two 16-byte words");

// Buffers of one round of the NEE_DS adjoint wavefront (vrt_wave_ds.cu).
struct WaveBw {
    ShadowJob* jobs;
    VertexRec* recs;
    CollisionRec* evs;         // the collision log
    float* info;               // per path: R (3), Rsp (3), first record, first collision (or kUnlogged)
    uint32_t* over;            // round-local indices of the paths left out of the log
    uint4* list;               // paths with logged collisions: round-local index, first collision, count
    // [0] jobs, [1] records, [2] re-walk queue, [3] / [4] heads of the shadow
    // kernels, [5] collisions, [6] paths left out of the log, [7] replay-list head,
    // [8] replay list
    unsigned long long* hdr;
    unsigned long long cap_jobs, cap_recs, cap_paths, cap_evs;
    unsigned long long res_jobs, res_recs, res_evs, lanes;
    uint64_t p_begin;
    // uncapped paths (max_bounces == 0): a path still going after kpass
    // vertices is handed to the state-machine adjoint (its global id into
    // spill, count in *spill_count); kpass == 0 with a bounce cap
    int kpass;
    unsigned long long* spill;
    unsigned long long* spill_count;
    unsigned long long cap_spill;
    // per path of the round: the DRT adjoint's reservoir (4 float4: vertex and
    // its weight, direction and the running total, throughput and the stream
    // position at the end of the primal), the DRTQ adjoint's segment 0 (3
    // float4, as in segs), or the SPS adjoint's entry point and
    // singular-vertex sigma (1 float4); null for NEE_DS
    float4* resv;
    // DRTQ: the segments after scattering vertices (3 float4 each: start and
    // length, direction and segment number, throughput and the path's index in
    // the round), *hdr[14] of them; null otherwise
    float4* segs;
    unsigned long long cap_segs;
};

// Path admission of the DRT and SPS primals (all lanes call it with the
// ballot of the lanes that want a path; the leader decides): new paths are
// taken while the round's buffers hold every lane's worst case, and each new
// path also gets one job slot (its primary ray's adjoint-only job).  Returns
// the warp's first path id (~0: no room this round) and, in jb, the first of
// those job slots.
__device__ __forceinline__ unsigned long long admit_paths(const WaveBw& wv, DScratch* sc, uint64_t n_paths,
                                                          unsigned want, unsigned long long& jb) {
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(want) - 1;
    unsigned long long base = 0;
    jb = 0;
    if ((int)lane == leader) {
        const unsigned long long uj = *((volatile unsigned long long*)&wv.hdr[0]);
        const unsigned long long ur = *((volatile unsigned long long*)&wv.hdr[1]);
        const unsigned long long ue = *((volatile unsigned long long*)&wv.hdr[5]);
        const unsigned long long up = *((volatile unsigned long long*)&sc->next_path) - wv.p_begin;
        const bool room = uj + wv.res_jobs <= wv.cap_jobs && ur + wv.res_recs <= wv.cap_recs &&
                          ue + wv.res_evs <= wv.cap_evs && up + wv.lanes <= wv.cap_paths;
        base = room ? atomicAdd(&sc->next_path, (unsigned long long)__popc(want)) : ~0ull;
        if (base != ~0ull && base < n_paths) {
            const unsigned long long nv =
                n_paths - base < (unsigned long long)__popc(want) ? n_paths - base : (unsigned long long)__popc(want);
            jb = atomicAdd(&wv.hdr[0], nv);
        }
    }
    jb = __shfl_sync(kAll, jb, leader);
    return __shfl_sync(kAll, base, leader);
}

}  // namespace wave

// The light jobs of the NEE_DS adjoint rounds (defined in vrt_wave.cu, so they
// are compiled with the forward's floating-point contraction): T of the
// primal's jobs into their vertex records and paths (head: hdr[3]; the DDA
// forms also run the DDA adjoint), and the ratio / delta tracking adjoints of
// the same jobs with dL/dT = dL/dR(pixel) / div . weight (head: hdr[4]).
int launch_shadow_record(const DMedium& M, const PathSrc& src, const wave::WaveBw& wv, uint64_t seed, const float* dL,
                         float div, DScratch* sc, int num_sms, cudaStream_t stream);
// mode ADJ_DRT / ADJ_SPS: the DRT or SPS adjoint's jobs (forks of stream 1,
// every job but those of handed-over paths, kAdjOnly jobs included; SPS: the
// rays after the singular vertex weighed by its sigma, wv.resv[k].w).
enum : int { ADJ_DS = 0, ADJ_DRT = 1, ADJ_SPS = 2 };
int launch_shadow_adjoint(const DMedium& M, const PathSrc& src, const wave::WaveBw& wv, uint64_t seed, const float* dL,
                          float div, DScratch* sc, int num_sms, cudaStream_t stream, int mode = ADJ_DS);

}  // namespace vrt
