// vrt_path.cu -- path integrators on sm_100a: forward passes and path-replay adjoints.
//
// Forward NEE integrator (include/vr_path_integrator_NEE.h:1-66) as a
// persistent state machine.  Every lane owns one path; one loop iteration
// performs ONE free-flight step of whatever segment the lane is in (the primary
// delta-tracking segment or a ratio/delta-tracking shadow segment), so the
// expensive part -- the sigma gather -- is executed by the whole warp together,
// and only the cheap event handling (collision, end of shadow ray, phase
// sampling) diverges.  When a lane's path ends, the warp refills all dead
// lanes at once from a global queue: one atomicAdd per warp per refill, ranks
// from a ballot.  Each lane consumes its path's Philox stream in exactly the
// order of the sequential definition, so results are independent of the
// schedule.
//
// The adjoints (NEE_DS, DT, NEE_DRT) replay each path from its Philox stream
// (path i re-derives every draw from (seed, i)), as the reference does from
// saved seeds, and scatter dL/dsigma and dL/dalbedo with atomics.
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_device.cuh"
#include "vrt_internal.h"
#include "vrt_tracking.cuh"

namespace vrt {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kPathStepCap = 1 << 26;  // total free-flight steps per path before VRT_E_ITER_CAP

__device__ __forceinline__ void primary_ray(const PathSrc& S, uint64_t pid, Rng& rng, float3& x, float3& w,
                                            long long& oidx) {
    if (S.is_camera) {
        long long p = (long long)(pid % (uint64_t)S.npix);
        camera_pixel_ray(S.cam, p, rng, x, w, nullptr);  // sensor triples are checked on the host
        oidx = p;
    } else {
        x = ld3(S.rays + 6 * pid);
        w = ld3(S.rays + 6 * pid + 3);
        oidx = (long long)pid;
    }
}

__device__ __forceinline__ void warp_add_counters(DScratch* sc, uint32_t paths, uint32_t verts, const Tally& tl) {
    unsigned long long p = paths, v = verts, s = tl.steps, l = tl.lookups, r = tl.reds, a = tl.albedo;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(kFull, p, o);
        v += __shfl_down_sync(kFull, v, o);
        s += __shfl_down_sync(kFull, s, o);
        l += __shfl_down_sync(kFull, l, o);
        r += __shfl_down_sync(kFull, r, o);
        a += __shfl_down_sync(kFull, a, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&sc->paths, p);
        atomicAdd(&sc->vertices, v);
        atomicAdd(&sc->steps, s);
        atomicAdd(&sc->lookups, l);
        atomicAdd(&sc->reds, r);
        atomicAdd(&sc->albedo, a);
    }
}

// ------------------------------------------------------------------------
// Forward NEE: persistent state machine.
// ------------------------------------------------------------------------
enum : int { ST_DEAD = 0, ST_PRIMARY = 1, ST_SHADOW = 2 };
enum : int { SH_DIRECT = 0, SH_ENV = 1, SH_SUN = 2 };
enum : int { EV_NONE = 0, EV_COLLISION = 1, EV_ESCAPE = 2, EV_SHADOW_DONE = 3 };

struct NeeLane {
    Flight ff;      // the current free flight (residual optical depth)
    Rng rng;        // the active stream: the path's, or a shadow ray's fork
    Rng park;       // the path's stream while a shadow ray runs
    bool parked;
    float3 x, w, W, R;
    float d;
    int bounces;
    float3 sx, sw;  // shadow segment position / direction
    float sd, T;
    float3 pay;     // radiance carried by the shadow ray
    float payph;    // phase value for it
    int kind;
    int state;
    long long oidx;
    uint32_t steps_path;
    long long pid;  // cache forms: the path's row
    int nrec;       // FW_TRAIN: collisions recorded so far
};

__device__ __forceinline__ void st3(float* p, float3 v) {
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
}

// A finished path: its estimate goes to the image / ray output.  A training
// path stores its estimate (the cache query, if any, is added later) and marks
// the collisions it never reached (NaN target, zero throughput).
template <int MODE>
__device__ __forceinline__ void end_path(const PathSrc& S, const NeeLane& L, float* out, float scale,
                                         const CacheIO& io) {
    if (MODE == FW_BRANCH) {  // the scattered-only path's estimate, per item
        st3(io.pR + 3 * L.oidx, L.R);
        return;
    }
    if (MODE == FW_TRAIN) {
        const long long n = io.rows * io.rec;
        st3(io.pR + 3 * L.pid, L.R);
        for (int k = L.nrec; k < io.rec; ++k) {
            float* o = io.smp + 3 * (L.pid * io.rec + k);
            st3(o, f3(0.0f));
            st3(o + 3 * n, make_float3(0.0f, 0.0f, 1.0f));
            st3(o + 6 * n, f3(__int_as_float(0x7fc00000)));
            st3(o + 9 * n, f3(0.0f));
        }
        return;
    }
    if (S.is_camera) {
        atomicAdd(out + 3 * L.oidx + 0, L.R.x * scale);
        atomicAdd(out + 3 * L.oidx + 1, L.R.y * scale);
        atomicAdd(out + 3 * L.oidx + 2, L.R.z * scale);
    } else {
        out[3 * L.oidx + 0] = L.R.x;
        out[3 * L.oidx + 1] = L.R.y;
        out[3 * L.oidx + 2] = L.R.z;
    }
}

// Begin a transmittance segment from x0 along dir (the transmittance map's own
// boundary test, vr_transmittance_RT.h:5-10 / _DT.h:3-8).  DDA segments are
// deterministic and evaluated inline.
__device__ __forceinline__ int start_shadow(const DMedium& M, NeeLane& L, float3 x0, float3 dir, Tally& tl) {
    L.state = ST_SHADOW;
    L.T = 1.0f;
    L.ff = Flight();
    Rng child = L.rng.fork();
    if (M.tr_mode >= 2) {  // DDA, GRT, GDT: one call
        if (M.tr_mode == 2) L.T = transmittance_dda<false>(M, x0, dir, tl);
        else if (M.tr_mode == 3) L.T = transmittance_dda<true>(M, x0, dir, tl);
        else if (M.tr_mode == 4) L.T = transmittance_grid_tracking<false>(M, child, x0, dir, tl, nullptr);
        else L.T = transmittance_grid_tracking<true>(M, child, x0, dir, tl, nullptr);
        return EV_SHADOW_DONE;
    }
    float tMin, tMax;
    if (!boundary(M, x0, dir, tMin, tMax)) return EV_SHADOW_DONE;
    L.sx = x0 + dir * tMin;
    L.sw = dir;
    L.sd = tMax - tMin;
    L.park = L.rng;
    L.rng = child;
    L.parked = true;
    return EV_NONE;
}

// vr_path_integrator_NEE.h:57-62 plus the optional bounce cap
__device__ __forceinline__ int after_nee(const DMedium& M, NeeLane& L) {
    ++L.bounces;
    if (M.max_bounces > 0 && L.bounces >= M.max_bounces) return EV_ESCAPE;
    float3 wo = phase_sample(M, L.rng, L.w);
    L.W = L.W * 1.0f;
    if (all_less(L.W, 0.00001f)) return EV_ESCAPE;
    L.w = wo;
    float tMin;
    boundary(M, L.x, L.w, tMin, L.d);
    L.ff = Flight();
    L.state = ST_PRIMARY;
    return L.d > 0.00001f ? EV_NONE : EV_ESCAPE;
}

// MODE: FW_PLAIN (the integrator), FW_CUT (unbiased prefix that stops into the
// radiance cache), FW_TRAIN (full paths from random pixels that record
// in-scattered radiance samples for the cache).
template <int MODE>
__global__ void __launch_bounds__(256, 3) k_nee_fw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed, float* out,
                                                 float scale, DScratch* sc, CacheIO io) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00001f;
    NeeLane L;
    L.state = ST_DEAD;
    bool exhausted = false;
    uint32_t n_paths_done = 0, n_verts = 0;
    Tally tl;

    while (true) {
        // ---- refill dead lanes from the global queue (one atomic per warp)
        unsigned want = __ballot_sync(kFull, L.state == ST_DEAD && !exhausted);
        if (want) {
            int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader)
                base = atomicAdd(MODE == FW_BRANCH ? io.queue : &sc->next_path, (unsigned long long)__popc(want));
            base = __shfl_sync(kFull, base, leader);
            if (L.state == ST_DEAD && !exhausted) {
                uint64_t pid = base + __popc(want & ((1u << lane) - 1u));
                if (pid >= n_paths) {
                    exhausted = true;
                } else {
                    // path_integrator_NEE prologue (vr_path_integrator_NEE.h:3-14)
                    float3 x0, w0;
                    if (MODE == FW_BRANCH) {  // a given start, on the stream where the caller left it
                        const float4 a = io.branch[3 * pid], b = io.branch[3 * pid + 1], c = io.branch[3 * pid + 2];
                        const uint64_t gp = (uint64_t)__float_as_uint(c.x) | ((uint64_t)__float_as_uint(c.y) << 32);
                        L.rng.init(seed, gp, __float_as_uint(c.z));
                        L.rng.seek(Rng::Pos{__float_as_uint(a.w), __float_as_uint(b.w)});
                        x0 = make_float3(a.x, a.y, a.z);
                        w0 = make_float3(b.x, b.y, b.z);
                        L.oidx = (long long)pid;
                    } else {
                        L.rng.init(seed, pid, 0);
                        if (MODE == FW_TRAIN && S.is_camera) {  // a random pixel: the path's first draw
                            const uint64_t px = ((uint64_t)L.rng.u32() * (uint64_t)S.npix) >> 32;
                            primary_ray(S, px, L.rng, x0, w0, L.oidx);
                        } else {
                            primary_ray(S, pid, L.rng, x0, w0, L.oidx);
                        }
                    }
                    L.pid = (long long)pid;
                    L.nrec = 0;
                    if (MODE == FW_CUT || (MODE == FW_TRAIN && io.cut >= 0)) {  // no query unless the path reaches the cut
                        float* q = io.q + 3 * L.pid;
                        st3(q, f3(0.0f));
                        st3(q + 3 * io.rows, make_float3(0.0f, 0.0f, 1.0f));
                        st3(q + 6 * io.rows, f3(0.0f));
                    }
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    L.x = x0 + w0 * tMin;
                    L.w = w0;
                    L.d = tMax - tMin;
                    L.W = f3(1.0f);
                    L.R = f3(0.0f);
                    L.bounces = 0;
                    L.steps_path = 0;
                    L.kind = SH_DIRECT;
                    L.parked = false;
                    ++n_paths_done;
                    if (MODE == FW_BRANCH) {  // scattered light only: no direct term
                        L.ff = Flight();
                        L.state = L.d > EPS ? ST_PRIMARY : ST_DEAD;
                        if (L.state == ST_DEAD) end_path<MODE>(S, L, out, scale, io);
                    } else {
                        int ev = start_shadow(M, L, L.x, L.w, tl);
                        if (ev == EV_SHADOW_DONE) {
                            L.R = L.R + L.T * env_radiance(M, L.w);
                            L.state = L.d > EPS ? ST_PRIMARY : ST_DEAD;
                            if (L.state == ST_DEAD) end_path<MODE>(S, L, out, scale, io);
                        }
                    }
                }
            }
        }
        if (__all_sync(kFull, L.state == ST_DEAD && exhausted)) break;
        if (L.state == ST_DEAD) continue;

        // ---- one free flight of the current segment; majorant-brick faces it
        // crosses are handled in the inner loop without new draws
        const bool prim = L.state == ST_PRIMARY;
        int ev = EV_NONE;
        bool need_sigma = false;
        float m = 0.0f, t = 0.0f;
        if (L.ff.tau < 0.0f) ++tl.steps;
        L.ff.sample(L.rng);
        for (int k = 0;; ++k) {
            if (k >= kStepCap) {
                raise_status(&sc->status, 4);
                ev = EV_ESCAPE;
                break;
            }
            float md;
            if (prim) {  // vr_path_integrator_NEE.h:20-33
                m = gmax(EPS, L.ff.bk.query(M, L.x, L.w, md));
                t = L.ff.tau / m;
                L.x = L.x + L.w * gmin(t, md);
                if (t > md) {
                    L.d -= md;
                    L.ff.cross(m, md);
                    L.ff.bk.advance(M);
                    if (!(L.d > EPS)) { ev = EV_ESCAPE; break; }
                    continue;
                }
                L.ff.used();
                if (t > L.d) ev = EV_ESCAPE;
                else need_sigma = true;
                L.ff.bk.move(t);
                break;
            } else if (M.tr_mode == 0) {  // vr_transmittance_RT.h:15-25
                m = gmax(0.0000001f, L.ff.bk.query(M, L.sx, L.sw, md));
                t = L.ff.tau / m;
                if (md < L.sd && t > md) {
                    L.sx = L.sx + L.sw * md;
                    L.sd -= md;
                    L.ff.cross(m, md);
                    L.ff.bk.advance(M);
                    continue;
                }
                L.ff.used();
                float dt = gmin(t, gmin(L.sd, md));
                L.ff.bk.move(dt);
                L.sx = L.sx + L.sw * dt;
                L.sd -= dt;
                if (L.sd <= 0.0000001f) ev = EV_SHADOW_DONE;
                else need_sigma = true;
                break;
            } else {  // vr_transmittance_DT.h:10-26
                m = gmax(0.0000001f, L.ff.bk.query(M, L.sx, L.sw, md));
                float dt = L.ff.tau / m;
                float tt = gmin(md, dt);
                L.sx = L.sx + L.sw * tt;
                L.sd -= tt;
                if (L.sd <= 0.0000001f) { L.ff.used(); ev = EV_SHADOW_DONE; break; }
                if (dt > md) { L.ff.cross(m, md); L.ff.bk.advance(M); continue; }
                L.ff.used();
                L.ff.bk.move(tt);
                need_sigma = true;
                break;
            }
        }
        if (need_sigma) {
            float s = sigma(M, prim ? L.x : L.sx, tl);
            if (prim) {
                if (L.rng.uniform() >= s / m) {
                    L.d -= t;
                    if (!(L.d > EPS)) ev = EV_ESCAPE;
                } else {
                    ev = EV_COLLISION;
                }
            } else if (M.tr_mode == 0) {
                L.T *= (1.0f - s / m);
                if (L.T < 0.01f) {
                    if (L.rng.uniform() < 1.0f - L.T) { L.T = 0.0f; ev = EV_SHADOW_DONE; }
                    else L.T = 1.0f;
                }
            } else {
                if (L.rng.uniform() < s / m) { L.T = 0.0f; ev = EV_SHADOW_DONE; }
            }
        }
        if (++L.steps_path > (uint32_t)kPathStepCap) {
            raise_status(&sc->status, 4);
            ev = EV_ESCAPE;
        }

        // ---- events (divergent, cheap)
        while (ev != EV_NONE) {
            if (ev == EV_COLLISION) {  // vr_path_integrator_NEE.h:41-50
                ++n_verts;
                if ((MODE == FW_CUT || (MODE == FW_TRAIN && io.cut >= 0)) && L.bounces == io.cut) {
                    // the rest of the path comes from the cache
                    float* q = io.q + 3 * L.pid;
                    st3(q, L.x);
                    st3(q + 3 * io.rows, L.w);
                    st3(q + 6 * io.rows, L.W);
                    ev = EV_ESCAPE;
                    continue;
                }
                if (MODE == FW_TRAIN && L.bounces < io.rec) {  // R and W at arrival; targets at the end
                    const long long n = io.rows * io.rec;
                    float* o = io.smp + 3 * (L.pid * io.rec + L.bounces);
                    st3(o, L.x);
                    st3(o + 3 * n, L.w);
                    st3(o + 6 * n, L.R);
                    st3(o + 9 * n, L.W);
                    L.nrec = L.bounces + 1;
                }
                float3 sa = albedo(M, L.x, tl);
                L.R = L.R + L.W * (f3(1.0f) - sa) * M.emission;
                L.W = L.W * sa;
                float3 wnee;
                L.pay = environment_sample(M, L.rng, wnee);
                L.payph = phase(M, L.w, wnee);
                L.kind = SH_ENV;
                ev = start_shadow(M, L, L.x, wnee, tl);
            } else if (ev == EV_SHADOW_DONE) {
                if (L.parked) {  // back to the path's stream
                    L.rng = L.park;
                    L.parked = false;
                }
                L.ff = Flight();
                if (L.kind == SH_DIRECT) {  // vr_path_integrator_NEE.h:13-14
                    L.R = L.R + L.T * env_radiance(M, L.w);
                    L.state = ST_PRIMARY;
                    ev = L.d > EPS ? EV_NONE : EV_ESCAPE;
                } else if (L.kind == SH_ENV) {  // :51-52
                    L.R = L.R + L.W * L.T * L.pay * L.payph;
                    if (M.has_sun) {
                        L.pay = M.sun_L;
                        L.payph = phase(M, L.w, M.sun_dir);
                        L.kind = SH_SUN;
                        ev = start_shadow(M, L, L.x, M.sun_dir, tl);
                    } else {
                        ev = after_nee(M, L);
                    }
                } else {
                    L.R = L.R + L.W * L.T * L.pay * L.payph;
                    ev = after_nee(M, L);
                }
            } else {  // EV_ESCAPE: the path's estimate is complete
                end_path<MODE>(S, L, out, scale, io);
                L.state = ST_DEAD;
                ev = EV_NONE;
            }
        }
    }
    warp_add_counters(sc, n_paths_done, n_verts, tl);
}

// ------------------------------------------------------------------------
// Sequential forms (one path per thread), used by the adjoints.
// ------------------------------------------------------------------------

// vr_path_integrator_NEE.h:1-66 (+ directional light, bounce cap)
__device__ float3 path_nee_seq(const DMedium& M, Rng& rng, float3 x, float3 w, bool only_scatters, uint32_t& verts,
                               Tally& tl, uint32_t* status) {
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    float3 R = f3(0.0f), W = f3(1.0f);
    if (!only_scatters) R = R + transmittance(M, rng, x, w, tl, status) * env_radiance(M, w);
    const float EPS = 0.00001f;
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); break; }
        float md;
        float m = gmax(EPS, ff.bk.query(M, x, w, md));
        if (ff.tau < 0.0f) ++tl.steps;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) { d -= t; continue; }
        ++verts;
        float3 sa = albedo(M, x, tl);
        R = R + W * (f3(1.0f) - sa) * M.emission;
        W = W * sa;
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        R = R + W * T_nee * env * phase(M, w, wnee);
        if (M.has_sun) {
            float T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            R = R + W * T_sun * M.sun_L * phase(M, w, M.sun_dir);
        }
        if (M.max_bounces > 0 && ++bounces >= M.max_bounces) return R;
        float3 wo = phase_sample(M, rng, w);
        if (all_less(W, EPS)) return R;
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
    }
    return R;
}

// vr_path_integrator_DT.h:59-235
__device__ void path_dt_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float eps, float3 dL_dR, Tally& tl,
                           uint32_t* status) {
    const Rng::Pos before_path = rng.pos();
    const float3 ini_x = x, ini_w = w;
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    const float EPS = 0.00000001f;
    float3 W = f3(1.0f);
    float null_W = 1.0f;
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps);
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        float Pc = (s + eps) / m;
        if (rng.uniform() >= Pc) { d -= t; W = W * ((1.0f - s / m) / (1.0f - Pc)); continue; }
        if (s == 0.0f) {
            if (null_W == 0.0f) { W = f3(0.0f); break; }
            null_W = 0.0f;
        } else {
            W = W * ((s / m) / Pc);
        }
        float3 sa = albedo(M, x, tl);
        float3 wo = phase_sample(M, rng, w);
        W = W * (sa * 1.0f);
        if (all_less(W, EPS)) { W = f3(0.0f); break; }
        if (M.max_bounces > 0 && ++bounces >= M.max_bounces) { W = f3(0.0f); break; }
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
    }
    const float3 dL_dW = dL_dR * env_radiance(M, w);
    rng.seek(before_path);
    x = ini_x;
    w = ini_w;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    d = tMax - tMin;
    const float3 W_out = W;
    W = f3(1.0f);
    bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps);
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        float Pc = (s + eps) / m;
        if (rng.uniform() >= Pc) {
            sigma_bw(M, x, dot(dL_dW, -W_out * null_W / m / (1.0f - s / m)), tl);
            W = W * ((1.0f - s / m) / (1.0f - Pc));
            d -= t;
            continue;
        }
        sigma_bw(M, x, dot(dL_dW, s == 0.0f ? W_out : W_out * null_W / s), tl);
        W = W * (s / m / Pc);
        if (s == 0.0f) break;
        float3 sa = albedo(M, x, tl);
        float3 wo = phase_sample(M, rng, w);
        W = W * sa;
        if (all_less(W, EPS)) return;
        if (M.max_bounces > 0 && ++bounces >= M.max_bounces) return;
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
    }
}

// vr_path_integrator_NEE_DS.h:6-206.  ds_compat selects the reference's
// replay majorant (x1.2 + 2 eps, different from its primal + 2 eps + 0.1);
// otherwise the replay uses the primal majorant and retraces the primal path.
__device__ void path_nee_ds_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float eps, float3 dL_dR,
                               Tally& tl, uint32_t* status) {
    const Rng::Pos before_path = rng.pos();
    const float3 ini_x = x, ini_w = w;
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    float3 R = f3(0.0f), R_after_sp = f3(0.0f), W = f3(1.0f);
    float null_W = 1.0f;
    const float EPS = 0.00000001f;
    bool scattered = false;
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps + 0.1f);
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        float Pc = (s + eps) / m;
        if (rng.uniform() >= Pc) { d -= t; W = W * ((1.0f - s / m) / (1.0f - Pc)); continue; }
        scattered = true;
        if (s < EPS) {
            if (null_W < EPS) { W = f3(0.0f); break; }
            null_W = 0.0f;
        } else {
            W = W * ((s / m) / Pc);
        }
        float3 sa = albedo(M, x, tl);
        float3 added_R = W * (f3(1.0f) - sa) * M.emission;
        W = W * sa;
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        added_R = added_R + W * T_nee * env * ph_nee;
        if (M.has_sun) {
            float T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            added_R = added_R + W * T_sun * M.sun_L * phase(M, w, M.sun_dir);
        }
        if (null_W < EPS) R_after_sp = R_after_sp + added_R;
        else R = R + added_R;
        if (M.max_bounces > 0 && ++bounces >= M.max_bounces) { W = f3(0.0f); break; }
        float3 wo = phase_sample(M, rng, w);
        if (all_less(W, EPS)) { W = f3(0.0f); break; }
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
    }
    if (!scattered) R = R + env_radiance(M, w) * W;

    rng.seek(before_path);
    x = ini_x;
    w = ini_w;
    W = f3(1.0f);
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    d = tMax - tMin;
    bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float mj = ff.bk.query(M, x, w, md);
        float m = M.ds_compat ? gmax(EPS, mj * 1.2f + 2.0f * eps) : gmax(EPS, mj + 2.0f * eps + 0.1f);
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        float Pc = (s + eps) / m;
        if (rng.uniform() >= Pc) {
            sigma_bw(M, x, dot(dL_dR, -R / m / (1.0f - s / m)), tl);
            W = W * ((1.0f - s / m) / (1.0f - Pc));
            d -= t;
            continue;
        }
        sigma_bw(M, x, dot(dL_dR, s < EPS ? R_after_sp / eps : R / s), tl);
        W = W * (s / m / Pc);
        if (s < EPS) return;
        float3 sa = albedo(M, x, tl);
        float3 dL_dsa = dL_dR * W * -1.0f * M.emission;
        R = R - W * (f3(1.0f) - sa) * M.emission;
        dL_dsa = dL_dsa + dL_dR * R / make_float3(gmax(EPS, sa.x), gmax(EPS, sa.y), gmax(EPS, sa.z));
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        const Rng::Pos before_tr = rng.pos();
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        const Rng::Pos before_sun = rng.pos();
        float T_sun = 0.0f, ph_sun = 0.0f;
        if (M.has_sun) {
            T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            ph_sun = phase(M, w, M.sun_dir);
        }
        float3 wo = phase_sample(M, rng, w);
        const Rng::Pos before_next = rng.pos();
        W = W * sa;
        float dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R = R - W * T_nee * env * ph_nee;
        float dL_dTsun = 0.0f;
        if (M.has_sun) {
            dL_dTsun = dot(dL_dR, W * M.sun_L * ph_sun);
            R = R - W * T_sun * M.sun_L * ph_sun;
        }
        albedo_bw(M, x, dL_dsa, tl);
        rng.seek(before_tr);
        transmittance_bw(M, rng, x, wnee, dL_dTnee, tl, status);
        if (M.has_sun) {
            rng.seek(before_sun);
            transmittance_bw(M, rng, x, M.sun_dir, dL_dTsun, tl, status);
        }
        rng.seek(before_next);
        if (M.max_bounces > 0 && ++bounces >= M.max_bounces) return;
        if (all_less(W, EPS)) return;
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
    }
}

// x + w t with the product and the sum each rounded (no contraction into an
// FMA): sample points of the position samplers land exactly on majorant-brick
// faces, where the brick chosen depends on the last bit.
__device__ __forceinline__ float3 ray_at(float3 x, float3 w, float t) {
    return make_float3(__fadd_rn(x.x, __fmul_rn(w.x, t)), __fadd_rn(x.y, __fmul_rn(w.y, t)),
                       __fadd_rn(x.z, __fmul_rn(w.z, t)));
}

// vr_path_integrator_NEE_DRT.h:8-60 sample_transmittance_position (majorant
// queried at the sample point x + w t)
__device__ float sample_transmittance_position(const DMedium& M, Rng& rng, float3 x, float3 w, float d, float& sample_t,
                                               float& weight_t, Tally& tl, uint32_t* status) {
    float Tr = 1.0f, t = 0.0f, res_t = 0.0f, res_dt = 0.0f, C = 0.0f;
    const float EPS = 0.0000001f;
    int it = 0;
    for (; it < kStepCap; ++it) {
        float md;
        float m = gmax(EPS, majorant(M, ray_at(x, w, t), w, md));
        float dt = gmin(-logf(1.0f - rng.uniform()) / m, gmin(md, d - t));
        float w_step = Tr * dt;
        C += w_step;
        if (rng.uniform() < w_step / C) { res_t = t; res_dt = dt; }
        t += dt;
        if (dt >= md - EPS) continue;
        if (t >= d - EPS) break;
        Tr *= 1.0f - sigma(M, ray_at(x, w, t), tl) / m;
    }
    if (it == kStepCap) raise_status(status, 4);
    weight_t = C;
    sample_t = res_t + rng.uniform() * res_dt;
    return Tr;
}

// vr_path_integrator_NEE_DRT.h:232-268: the branch from the reservoir vertex
// (res_x, res_w, throughput res_W picked with weight res_P of total_weight) --
// a transmittance-sampled position, its light rays and a nested scattered-only
// NEE path -- and its sigma scatter.  rng is the path's stream where the
// replay left it (the primal's end).
__device__ void drt_branch(const DMedium& M, Rng& rng, float3 res_x, float3 res_w, float3 res_W, float res_P,
                           float total_weight, float3 dL_dR, uint32_t& verts, Tally& tl, uint32_t* status) {
    float tMin, d;
    boundary(M, res_x, res_w, tMin, d);
    float s_t, weight_t;
    sample_transmittance_position(M, rng, res_x, res_w, d, s_t, weight_t, tl, status);
    float3 xs = res_x + res_w * s_t;
    float3 ls_dir;
    float3 Ls_env = environment_sample(M, rng, ls_dir);
    float3 Ls = transmittance(M, rng, xs, ls_dir, tl, status) * Ls_env * phase(M, res_w, ls_dir);
    if (M.has_sun) Ls = Ls + transmittance(M, rng, xs, M.sun_dir, tl, status) * M.sun_L * phase(M, res_w, M.sun_dir);
    float3 ws = phase_sample(M, rng, res_w);
    Ls = Ls + 1.0f * path_nee_seq(M, rng, xs, ws, true, verts, tl, status);
    Ls = Ls * res_W * weight_t * albedo(M, xs, tl);
    float sigma_xs = sigma(M, xs, tl);
    float mis_T = 1.0f / (1.0f + sigma_xs * sigma_xs);
    sigma_bw(M, xs, dot(dL_dR, Ls) * mis_T * total_weight / res_P, tl);
}

// vr_path_integrator_NEE_DRT.h:62-270.  The branch seed is Philox stream 1.
__device__ void path_nee_drt_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float3 dL_dR, Tally& tl,
                                uint32_t* status) {
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    if (d <= 0.0f) return;
    Rng sec;
    sec.k0 = rng.k0; sec.k1 = rng.k1; sec.plo = rng.plo; sec.phi = rng.phi;
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    uint32_t verts = 0;
    (void)transmittance(M, rng, x, w, tl, status);
    transmittance_bw(M, sec, x, w, dot(dL_dR, env_radiance(M, w)), tl, status);
    float3 R = f3(0.0f), W = f3(1.0f);
    float3 res_x = x, res_w = w, res_W = W;
    float res_P = 3.0f, total_weight = 3.0f;
    const float3 ini_x = x, ini_w = w;
    const float ini_d = d;
    const float EPS = 0.00000001f;
    const Rng::Pos before_path = rng.pos();
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) { d -= t; continue; }
        float3 sa = albedo(M, x, tl);
        W = W * sa;
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        R = R + W * T_nee * env * ph_nee;
        if (M.has_sun) {
            float T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            R = R + W * T_sun * M.sun_L * phase(M, w, M.sun_dir);
        }
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        float3 wo = phase_sample(M, rng, w);
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        float current_P = W.x + W.y + W.z;
        total_weight += current_P;
        if (rng.uniform() < current_P / total_weight) {
            res_P = current_P; res_W = W; res_x = x; res_w = w;
        }
        if (all_less(W, EPS) || capped) break;
    }
    W = f3(1.0f);
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng.seek(before_path);
    bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) {
            sigma_bw(M, x, dot(dL_dR, -R / m / (1.0f - s / m)), tl);
            d -= t;
            continue;
        }
        float mis_Ts = s * s / (1.0f + s * s);
        float dL_dsigma = dot(dL_dR, mis_Ts * R / s);
        float3 sa = albedo(M, x, tl);
        W = W * sa;
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        float T_sun = 0.0f, ph_sun = 0.0f;
        if (M.has_sun) {
            T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            ph_sun = phase(M, w, M.sun_dir);
        }
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        float3 wo = phase_sample(M, rng, w);
        float dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R = R - W * T_nee * env * ph_nee;
        float dL_dTsun = 0.0f;
        if (M.has_sun) {
            dL_dTsun = dot(dL_dR, W * M.sun_L * ph_sun);
            R = R - W * T_sun * M.sun_L * ph_sun;
        }
        sigma_bw(M, x, dL_dsigma, tl);
        transmittance_bw(M, sec, x, wnee, dL_dTnee, tl, status);
        if (M.has_sun) transmittance_bw(M, sec, x, M.sun_dir, dL_dTsun, tl, status);
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        rng.advance();
        if (all_less(W, EPS) || capped) break;
    }
    drt_branch(M, rng, res_x, res_w, res_W, res_P, total_weight, dL_dR, verts, tl, status);
}

__device__ __forceinline__ Rng branch_stream(const Rng& rng) {
    Rng sec;
    sec.k0 = rng.k0; sec.k1 = rng.k1; sec.plo = rng.plo; sec.phi = rng.phi;
    sec.stream = rng.stream + 1;
    sec.n = 0;
    sec.ntr = 0;
    return sec;
}

// vr_path_integrator_NEE_DRTQ.h:45-55 in_scattering (+ directional light)
__device__ float3 in_scattering(const DMedium& M, Rng& rng, float3 x, float3 w, Tally& tl, uint32_t* status) {
    float3 ls_dir;
    float3 Ls_env = environment_sample(M, rng, ls_dir);
    float3 Ls = transmittance(M, rng, x, ls_dir, tl, status) * Ls_env * phase(M, w, ls_dir);
    if (M.has_sun) Ls = Ls + transmittance(M, rng, x, M.sun_dir, tl, status) * M.sun_L * phase(M, w, M.sun_dir);
    float3 ws = phase_sample(M, rng, w);
    uint32_t verts = 0;
    Ls = Ls + 1.0f * path_nee_seq(M, rng, x, ws, true, verts, tl, status);
    return albedo(M, x, tl) * Ls;
}

// scatter-gradient term of a segment (_DRTQ.h:156-165, :249-259) on the
// segment's own stream (Rng::segment_stream)
__device__ void drtq_scatter_term(const DMedium& M, Rng sec, float3 x, float3 w, float d, float3 W, float3 dL_dR,
                                  Tally& tl, uint32_t* status) {
    float s_t, weight_t;
    sample_transmittance_position(M, sec, x, w, d, s_t, weight_t, tl, status);
    float3 xs = x + w * s_t;
    float3 Ls = in_scattering(M, sec, xs, w, tl, status);
    float sigma_t = sigma(M, xs, tl);
    float mis_T = 1.0f / (1.0f + sigma_t * sigma_t);
    sigma_bw(M, xs, mis_T * weight_t * dot(dL_dR, W * Ls), tl);
}

// vr_path_integrator_NEE_DRTQ.h:58-260.  The light rays' adjoints take fork j
// of stream 1 beside fork j of the path's stream (as in DRT); each segment's
// scatter term draws from its own stream, so the wavefront form can run them
// as independent items.  A path stops at 2^24 - 1 segments (error 4).
__device__ void path_nee_drtq_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float3 dL_dR, Tally& tl,
                                 uint32_t* status) {
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    if (d <= 0.0f) return;
    Rng sec = branch_stream(rng);
    (void)transmittance(M, rng, x, w, tl, status);
    transmittance_bw(M, sec, x, w, dot(dL_dR, env_radiance(M, w)), tl, status);
    float3 R = f3(0.0f), W = f3(1.0f);
    const float3 ini_x = x, ini_w = w;
    const float ini_d = d;
    const float EPS = 0.00000001f;
    const Rng::Pos before_path = rng.pos();
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) { d -= t; continue; }
        W = W * albedo(M, x, tl);
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        R = R + W * T_nee * env * phase(M, w, wnee);
        if (M.has_sun) R = R + W * transmittance(M, rng, x, M.sun_dir, tl, status) * M.sun_L * phase(M, w, M.sun_dir);
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        w = phase_sample(M, rng, w);
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        if (all_less(W, EPS) || capped) break;
    }
    W = f3(1.0f);
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng.seek(before_path);
    bounces = 0;
    uint32_t vertex = 0;  // scattering vertices so far: the next segment's number
    drtq_scatter_term(M, rng.segment_stream(0), x, w, d, W, dL_dR, tl, status);
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) {
            sigma_bw(M, x, dot(dL_dR, -R / m / (1.0f - s / m)), tl);
            d -= t;
            continue;
        }
        float dL_dsigma = dot(dL_dR, s * s / (1.0f + s * s) * R / s);
        W = W * albedo(M, x, tl);
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        float T_sun = 0.0f, ph_sun = 0.0f;
        if (M.has_sun) {
            T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            ph_sun = phase(M, w, M.sun_dir);
        }
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        float3 wo = phase_sample(M, rng, w);
        float dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R = R - W * T_nee * env * ph_nee;
        float dL_dTsun = 0.0f;
        if (M.has_sun) {
            dL_dTsun = dot(dL_dR, W * M.sun_L * ph_sun);
            R = R - W * T_sun * M.sun_L * ph_sun;
        }
        sigma_bw(M, x, dL_dsigma, tl);
        transmittance_bw(M, sec, x, wnee, dL_dTnee, tl, status);
        if (M.has_sun) transmittance_bw(M, sec, x, M.sun_dir, dL_dTsun, tl, status);
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        if (all_less(W, EPS) || capped) break;
        if (++vertex + 1u >= (1u << 24)) { raise_status(status, 4); return; }
        drtq_scatter_term(M, rng.segment_stream(vertex), x, w, d, W, dL_dR, tl, status);
    }
}

// vr_path_integrator_NEE_DRTDS.h:8-38 (majorant at the sample point)
__device__ void sample_collision_position_ds(const DMedium& M, Rng& rng, float3 x, float3 w, float d, float epsilon,
                                             float& t, float& weight_t, Tally& tl, uint32_t* status) {
    const float EPS = 0.0000001f;
    t = 0.0f;
    weight_t = 1.0f;
    for (int it = 0; it < kStepCap; ++it) {
        float md;
        float m = gmax(EPS, majorant(M, ray_at(x, w, t), w, md) + 2.0f * epsilon + 0.1f);
        float dt = gmin(-logf(1.0f - rng.uniform()) / m, gmin(md, d - t));
        t += dt;
        if (dt >= md - EPS) continue;
        if (t >= d - EPS) { weight_t = 0.0f; return; }
        float s = sigma(M, ray_at(x, w, t), tl);
        float Pc = (s + epsilon) / m;
        if (rng.uniform() < Pc) {
            weight_t *= 1.0f / (s + epsilon);
            return;
        }
        weight_t *= (1.0f - s / m) / (1.0f - Pc);
    }
    raise_status(status, 4);
    weight_t = 0.0f;
}

// vr_path_integrator_NEE_DRTDS.h:230-252: the branch from the reservoir vertex
// with a defensively sampled collision position (no MIS weight).
__device__ void drtds_branch(const DMedium& M, Rng& rng, float3 res_x, float3 res_w, float3 res_W, float res_P,
                             float total_weight, float epsilon, float3 dL_dR, uint32_t& verts, Tally& tl,
                             uint32_t* status) {
    float tMin, d;
    boundary(M, res_x, res_w, tMin, d);
    float s_t, weight_t;
    sample_collision_position_ds(M, rng, res_x, res_w, d, epsilon, s_t, weight_t, tl, status);
    if (weight_t > 0.0f) {
        float3 xs = res_x + res_w * s_t;
        float3 ls_dir;
        float3 Ls_env = environment_sample(M, rng, ls_dir);
        float3 Ls = transmittance(M, rng, xs, ls_dir, tl, status) * Ls_env * phase(M, res_w, ls_dir);
        if (M.has_sun) Ls = Ls + transmittance(M, rng, xs, M.sun_dir, tl, status) * M.sun_L * phase(M, res_w, M.sun_dir);
        float3 ws = phase_sample(M, rng, res_w);
        Ls = Ls + 1.0f * path_nee_seq(M, rng, xs, ws, true, verts, tl, status);
        Ls = Ls * res_W * weight_t * albedo(M, xs, tl);
        sigma_bw(M, xs, dot(dL_dR, Ls) * total_weight / res_P, tl);
    }
}

// vr_path_integrator_NEE_DRTDS.h:40-253 (branch seed = Philox stream 1)
__device__ void path_nee_drtds_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float epsilon, float3 dL_dR,
                                  Tally& tl, uint32_t* status) {
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    if (d <= 0.0f) return;
    Rng sec = branch_stream(rng);
    uint32_t verts = 0;
    (void)transmittance(M, rng, x, w, tl, status);
    transmittance_bw(M, sec, x, w, dot(dL_dR, env_radiance(M, w)), tl, status);
    float3 R = f3(0.0f), W = f3(1.0f);
    float3 res_x = x, res_w = w, res_W = W;
    float res_P = 3.0f, total_weight = 3.0f;
    const float3 ini_x = x, ini_w = w;
    const float ini_d = d;
    const float EPS = 0.00000001f;
    const Rng::Pos before_path = rng.pos();
    int bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) { d -= t; continue; }
        W = W * albedo(M, x, tl);
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        R = R + W * T_nee * env * phase(M, w, wnee);
        if (M.has_sun) R = R + W * transmittance(M, rng, x, M.sun_dir, tl, status) * M.sun_L * phase(M, w, M.sun_dir);
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        w = phase_sample(M, rng, w);
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        float current_P = W.x + W.y + W.z;
        total_weight += current_P;
        if (rng.uniform() < current_P / total_weight) {
            res_P = current_P; res_W = W; res_x = x; res_w = w;
        }
        if (all_less(W, EPS) || capped) break;
    }
    W = f3(1.0f);
    x = ini_x;
    w = ini_w;
    d = ini_d;
    rng.seek(before_path);
    bounces = 0;
    for (Flight ff; d > EPS; ++ff.it) {
        if (ff.it >= kPathStepCap) { raise_status(status, 4); return; }
        float md;
        float m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
        float t = ff.sample(rng) / m;
        x = x + w * gmin(t, md);
        if (t > md) { d -= md; ff.cross(m, md); ff.bk.advance(M); continue; }
        ff.used();
        if (t > d) break;
        ff.bk.move(t);
        float s = sigma(M, x, tl);
        if (rng.uniform() >= s / m) {
            sigma_bw(M, x, dot(dL_dR, -R / m / (1.0f - s / m)), tl);
            d -= t;
            continue;
        }
        float3 sa = albedo(M, x, tl);
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        float T_sun = 0.0f, ph_sun = 0.0f;
        if (M.has_sun) {
            T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            ph_sun = phase(M, w, M.sun_dir);
        }
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        float3 wo = phase_sample(M, rng, w);
        W = W * sa;
        float dL_dTnee = dot(dL_dR, W * env * ph_nee);
        R = R - W * T_nee * env * ph_nee;
        float dL_dTsun = 0.0f;
        if (M.has_sun) {
            dL_dTsun = dot(dL_dR, W * M.sun_L * ph_sun);
            R = R - W * T_sun * M.sun_L * ph_sun;
        }
        transmittance_bw(M, sec, x, wnee, dL_dTnee, tl, status);
        if (M.has_sun) transmittance_bw(M, sec, x, M.sun_dir, dL_dTsun, tl, status);
        w = wo;
        boundary(M, x, w, tMin, d);
        ff.bk.reset();
        rng.advance();
        if (all_less(W, EPS) || capped) break;
    }
    drtds_branch(M, rng, res_x, res_w, res_W, res_P, total_weight, epsilon, dL_dR, verts, tl, status);
}

// vr_path_integrator_NEE_SPS.h:1-59 (majorant at the current sample point;
// pow(sigma, 3) as sigma * sigma * sigma)
__device__ bool sample_collision_position(const DMedium& M, Rng& rng, float3 x, float3 w, float d, float3& xc,
                                          float& weight_xc, float& sigma_xc, int& samples, bool& mis_allowed,
                                          Tally& tl, uint32_t* status) {
    float t = 0.0f;
    weight_xc = 0.0f;
    sigma_xc = 0.0f;
    samples = 0;
    xc = x;
    int it = 0;
    for (; it < kStepCap; ++it) {
        float md;
        float m = majorant(M, xc, w, md) + 0.000001f;
        float dt = gmin(-logf(1.0f - rng.uniform()) / m, gmin(md, d - t));
        t += dt;
        xc = ray_at(x, w, t);
        if (dt >= md - 0.0000001f) continue;
        if (t >= d - 0.0000001f) break;
        float s = sigma(M, xc, tl);
        samples++;
        if (rng.uniform() < s / m) {
            weight_xc = 1.0f;
            sigma_xc = s;
            break;
        }
    }
    if (it == kStepCap) raise_status(status, 4);
    if (!mis_allowed) return false;
    float powered_c = sigma_xc * sigma_xc * sigma_xc;
    float mis_wc = weight_xc * powered_c / (1.0f + powered_c);
    float u = rng.uniform();
    float3 xf = xc * (1.0f - u) + x * u;
    float sigma_f = sigma(M, xf, tl);
    float powered_f = sigma_f * sigma_f * sigma_f;
    float mis_wf = t / (1.0f + powered_f);
    weight_xc = mis_wc + mis_wf;
    if (rng.uniform() * weight_xc < mis_wf) {
        xc = xf;
        sigma_xc = sigma_f;
        mis_allowed = false;
        return true;
    }
    return false;
}

// vr_path_integrator_NEE_SPS.h:88-101 st_tau_bw (stratified bins)
__device__ void st_tau_bw(const DMedium& M, Rng& rng, float3 a, float3 b, int bins, float dL_dtau, Tally& tl) {
    if (dL_dtau == 0.0f || bins == 0) return;
    float d = sqrtf(dot(a - b, a - b));
    float g = dL_dtau * d / (float)bins;
    for (int i = 0; i < bins; ++i) {
        float f = ((float)i + rng.uniform()) / (float)bins;
        sigma_bw(M, b * (1.0f - f) + a * f, g, tl);
    }
}

// vr_path_integrator_NEE_SPS.h:104-263 (emission ignored, as in the reference)
__device__ void path_nee_sps_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float3 dL_dR, Tally& tl,
                                uint32_t* status) {
    float tMin, tMax;
    boundary(M, x, w, tMin, tMax);
    x = x + w * tMin;
    float d = tMax - tMin;
    if (d <= 0.0f) return;
    Rng sec = branch_stream(rng);
    (void)transmittance(M, rng, x, w, tl, status);
    transmittance_bw(M, sec, x, w, dot(dL_dR, env_radiance(M, w)), tl, status);
    float3 R = f3(0.0f), Rf = f3(0.0f), W = f3(1.0f);
    float W_singular = 1.0f;
    bool mis_allowed = true;
    const float3 ini_x = x, ini_w = w;
    const float ini_d = d;
    const float EPS = 0.00001f;
    const Rng::Pos before_path = rng.pos();
    int bounces = 0;
    for (int it = 0; it < kStepCap; ++it) {
        float weight_xc, sigma_xc;
        float3 xc;
        int samples;
        if (sample_collision_position(M, rng, x, w, d, xc, weight_xc, sigma_xc, samples, mis_allowed, tl, status))
            W_singular = sigma_xc;
        if (weight_xc == 0.0f) break;
        x = xc;
        W = W * (weight_xc * albedo(M, x, tl));
        float3 wnee;
        float3 nee_env = environment_sample(M, rng, wnee);
        float nee_T = transmittance(M, rng, x, wnee, tl, status);
        float3 added_R = W * nee_T * phase(M, w, wnee) * nee_env;
        if (M.has_sun) added_R = added_R + W * transmittance(M, rng, x, M.sun_dir, tl, status) * phase(M, w, M.sun_dir) * M.sun_L;
        if (mis_allowed) R = R + added_R;
        else Rf = Rf + added_R;
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        w = phase_sample(M, rng, w);
        boundary(M, x, w, tMin, d);
        if (all_less(W, EPS) || capped) break;
    }
    W = f3(1.0f);
    mis_allowed = true;
    x = ini_x;
    w = ini_w;
    d = ini_d;
    float3 prev_x = x;
    rng.seek(before_path);
    bounces = 0;
    for (int it = 0; it < kStepCap; ++it) {
        float weight_xc, sigma_xc;
        float3 xc;
        int samples;
        bool singular = sample_collision_position(M, rng, x, w, d, xc, weight_xc, sigma_xc, samples, mis_allowed, tl,
                                                  status);
        if (weight_xc == 0.0f) break;
        float3 further_R = R + W_singular * Rf;
        float k = dot(dL_dR, further_R);
        float dL_dtau = -k;
        float dL_dsigma = singular ? dot(dL_dR, Rf) : k / gmax(0.001f, sigma_xc);
        x = xc;
        W = W * weight_xc;
        W = W * albedo(M, x, tl);
        float3 wnee;
        float3 env = environment_sample(M, rng, wnee);
        float T_nee = transmittance(M, rng, x, wnee, tl, status);
        float ph_nee = phase(M, w, wnee);
        float T_sun = 0.0f, ph_sun = 0.0f;
        if (M.has_sun) {
            T_sun = transmittance(M, rng, x, M.sun_dir, tl, status);
            ph_sun = phase(M, w, M.sun_dir);
        }
        bool capped = M.max_bounces > 0 && ++bounces >= M.max_bounces;
        float3 wo = phase_sample(M, rng, w);
        const float fs = mis_allowed ? 1.0f : W_singular;
        float dL_dTnee = dot(dL_dR, W * fs * env * ph_nee);
        float3 added_R = W * T_nee * ph_nee * env;
        float dL_dTsun = 0.0f;
        if (M.has_sun) {
            dL_dTsun = dot(dL_dR, W * fs * M.sun_L * ph_sun);
            added_R = added_R + W * T_sun * ph_sun * M.sun_L;
        }
        if (mis_allowed) R = R - added_R;
        else Rf = Rf - added_R;
        sigma_bw(M, x, dL_dsigma, tl);
        st_tau_bw(M, sec, x, prev_x, samples > 1 ? samples : 1, dL_dtau, tl);
        transmittance_bw(M, sec, x, wnee, dL_dTnee, tl, status);
        if (M.has_sun) transmittance_bw(M, sec, x, M.sun_dir, dL_dTsun, tl, status);
        w = wo;
        boundary(M, x, w, tMin, d);
        if (all_less(W, EPS) || capped) break;
        prev_x = x;
    }
}

// ------------------------------------------------------------------------
// Kernels over paths: the DT forms as persistent state machines, the other
// adjoints one path per thread (grid-stride)
// ------------------------------------------------------------------------

// The DT forward (vr_path_integrator_DT.h:7-57) as a persistent
// state machine: one free flight (at most 12 brick crossings, then a
// collision) per lane and iteration, lanes refilled by ballot.
__global__ void __launch_bounds__(256, 3) k_dt_fw_sm(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed, float* out,
                                                   float scale, DScratch* sc) {
    constexpr int kCrossIt = 12;  // brick crossings per iteration
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f), R = f3(0.0f);
    float d = 0.0f;
    int bounces = 0;
    bool alive = false, exhausted = false;
    long long oidx = 0;
    uint32_t paths = 0, verts = 0, steps_path = 0;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kFull, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
            base = __shfl_sync(kFull, base, leader);
            if (!alive && !exhausted) {
                const uint64_t pid = base + __popc(want & ((1u << lane) - 1u));
                if (pid >= n_paths) {
                    exhausted = true;
                } else {
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    primary_ray(S, pid, rng, x0, w0, oidx);
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    x = x0 + w0 * tMin;
                    w = w0;
                    d = tMax - tMin;
                    W = f3(1.0f);
                    R = f3(0.0f);
                    bounces = 0;
                    steps_path = 0;
                    ff = Flight();
                    alive = true;
                    ++paths;
                }
            }
        }
        if (__all_sync(kFull, !alive && exhausted)) break;
        if (!alive) continue;
        int ev = 0;  // 0 going on, 1 escaped (W * env + R), 2 ended (R)
        if (!(d > EPS)) {
            ev = 1;
        } else {
            float m = 0.0f, t = 0.0f;
            bool need = false;
            for (int k = 0;; ++k) {
                float md;
                m = gmax(EPS, ff.bk.query(M, x, w, md));
                if (ff.tau < 0.0f) ++tl.steps;
                t = ff.sample(rng) / m;
                x = x + w * gmin(t, md);
                if (t > md) {
                    d -= md;
                    ff.cross(m, md);
                    ff.bk.advance(M);
                    if (!(d > EPS)) { ev = 1; break; }
                    if (k + 1 >= kCrossIt) break;  // the flight resumes in the next iteration
                    continue;
                }
                ff.used();
                if (t > d) {
                    ev = 1;
                } else {
                    need = true;
                    ff.bk.move(t);
                }
                break;
            }
            if (need) {
                const float s = sigma(M, x, tl);
                if (rng.uniform() >= s / m) {
                    d -= t;
                    if (!(d > EPS)) ev = 1;
                } else {  // a real collision (_DT.h:39-52)
                    ++verts;
                    const float3 sa = albedo(M, x, tl);
                    R = R + W * (f3(1.0f) - sa) * M.emission;
                    W = W * sa;
                    const float3 wo = phase_sample(M, rng, w);
                    if (all_less(W, 0.0000001f) || (M.max_bounces > 0 && ++bounces >= M.max_bounces)) {
                        ev = 2;
                    } else {
                        w = wo;
                        float tMin;
                        boundary(M, x, w, tMin, d);
                        ff.bk.reset();
                    }
                }
            }
        }
        if (++steps_path > (uint32_t)kPathStepCap) {
            raise_status(&sc->status, 4);
            ev = 1;  // (the reference's loop ends with the escape term)
        }
        if (ev) {
            if (ev == 1) R = W * env_radiance(M, w) + R;
            if (S.is_camera) {
                atomicAdd(out + 3 * oidx + 0, R.x * scale);
                atomicAdd(out + 3 * oidx + 1, R.y * scale);
                atomicAdd(out + 3 * oidx + 2, R.z * scale);
            } else {
                out[3 * oidx + 0] = R.x;
                out[3 * oidx + 1] = R.y;
                out[3 * oidx + 2] = R.z;
            }
            alive = false;
        }
    }
    warp_add_counters(sc, paths, verts, tl);
}

// The DT adjoint (path_dt_bw, vr_path_integrator_DT.h:59-150) as a persistent
// state machine: every lane advances its path by one free flight per
// iteration -- at most 12 brick crossings, then a collision -- first through
// the primal walk, then through the replay of the same draws, and takes a new
// path when both are done (warp refill by ballot, one atomic per warp), so
// lanes do not wait for the longest path of their warp.  The replay restarts
// from the primary ray, drawn again from the path's stream; the arithmetic is
// path_dt_bw's, operation for operation.
__global__ void __launch_bounds__(256, 3) k_dt_bw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                const float* __restrict__ dL, float div, DScratch* sc) {
    constexpr int kCrossIt = 12;  // brick crossings per iteration
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f), W_out = f3(0.0f), dL_dW = f3(0.0f);
    float d = 0.0f, null_W = 1.0f;
    int bounces = 0, phase = 0;  // 0 idle, 1 primal, 2 replay
    bool exhausted = false;
    uint64_t pid = 0;
    uint32_t paths = 0, steps_path = 0;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kFull, phase == 0 && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
            base = __shfl_sync(kFull, base, leader);
            if (phase == 0 && !exhausted) {
                const uint64_t p = base + __popc(want & ((1u << lane) - 1u));
                if (p >= n_paths) {
                    exhausted = true;
                } else {
                    pid = p;
                    phase = 1;
                    null_W = 1.0f;
                    steps_path = 0;
                    ++paths;
                }
            }
        }
        if (__all_sync(kFull, phase == 0 && exhausted)) break;
        if (phase == 0) continue;
        if (steps_path == 0) {  // the start of a walk: the primary ray (the replay draws it again)
            rng.init(seed, pid, 0);
            long long oidx;
            float3 x0, w0;
            primary_ray(S, pid, rng, x0, w0, oidx);
            if (phase == 1) dL_dW = ld3(dL + 3 * oidx) / div;  // dL/dR for now; times the escape radiance below
            float tMin, tMax;
            boundary(M, x0, w0, tMin, tMax);
            x = x0 + w0 * tMin;
            w = w0;
            d = tMax - tMin;
            W = f3(1.0f);
            bounces = 0;
            ff = Flight();
        }
        bool end = !(d > EPS);
        if (!end) {
            float m = 0.0f, t = 0.0f;
            bool need = false;
            for (int k = 0;; ++k) {
                float md;
                m = gmax(EPS, ff.bk.query(M, x, w, md) + 2.0f * eps);
                if (ff.tau < 0.0f) ++tl.steps;
                t = ff.sample(rng) / m;
                x = x + w * gmin(t, md);
                if (t > md) {
                    d -= md;
                    ff.cross(m, md);
                    ff.bk.advance(M);
                    if (!(d > EPS)) { end = true; break; }
                    if (k + 1 >= kCrossIt) break;  // the flight resumes in the next iteration
                    continue;
                }
                ff.used();
                if (t > d) end = true;
                else need = true;
                if (need) ff.bk.move(t);
                break;
            }
            if (need) {
                const float s = sigma(M, x, tl);
                const float Pc = (s + eps) / m;
                if (rng.uniform() >= Pc) {  // null collision
                    if (phase == 2) sigma_bw(M, x, dot(dL_dW, -W_out * null_W / m / (1.0f - s / m)), tl);
                    d -= t;
                    W = W * ((1.0f - s / m) / (1.0f - Pc));
                    if (!(d > EPS)) end = true;
                } else if (phase == 1) {  // real collision of the primal (_DT.h:82-101)
                    bool stop = false;
                    if (s == 0.0f) {
                        if (null_W == 0.0f) { W = f3(0.0f); stop = true; }
                        else null_W = 0.0f;
                    } else {
                        W = W * ((s / m) / Pc);
                    }
                    if (!stop) {
                        const float3 sa = albedo(M, x, tl);
                        const float3 wo = phase_sample(M, rng, w);
                        W = W * (sa * 1.0f);
                        if (all_less(W, EPS)) { W = f3(0.0f); stop = true; }
                        else if (M.max_bounces > 0 && ++bounces >= M.max_bounces) { W = f3(0.0f); stop = true; }
                        else {
                            w = wo;
                            float tMin;
                            boundary(M, x, w, tMin, d);
                            ff.bk.reset();
                        }
                    }
                    if (stop) end = true;
                } else {  // real collision of the replay (_DT.h:125-148)
                    sigma_bw(M, x, dot(dL_dW, s == 0.0f ? W_out : W_out * null_W / s), tl);
                    W = W * (s / m / Pc);
                    if (s == 0.0f) {
                        end = true;
                    } else {
                        const float3 sa = albedo(M, x, tl);
                        const float3 wo = phase_sample(M, rng, w);
                        W = W * sa;
                        if (all_less(W, EPS) || (M.max_bounces > 0 && ++bounces >= M.max_bounces)) {
                            end = true;
                        } else {
                            w = wo;
                            float tMin;
                            boundary(M, x, w, tMin, d);
                            ff.bk.reset();
                        }
                    }
                }
            }
        }
        if (++steps_path > (uint32_t)kPathStepCap) {
            raise_status(&sc->status, 4);
            phase = 0;  // abandoned (the error word reports it)
            continue;
        }
        if (end) {
            if (phase == 1) {  // the primal's end: the escape radiance's weight, then the replay
                dL_dW = dL_dW * env_radiance(M, w);
                W_out = W;
                phase = 2;
                steps_path = 0;
            } else {
                phase = 0;
            }
        }
    }
    warp_add_counters(sc, paths, 0, tl);
}

// pids: the n_paths paths listed there (device array), else paths 0 .. n_paths-1
template <int MODE>
__global__ void __launch_bounds__(256) k_path_bw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed, const float* dL,
                                                  float div, DScratch* sc, const unsigned long long* pids) {
    uint32_t paths = 0;
    Tally tl;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_paths;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pid = pids ? (uint64_t)pids[i] : i;
        Rng rng;
        rng.init(seed, pid, 0);
        float3 x, w;
        long long oidx;
        primary_ray(S, pid, rng, x, w, oidx);
        float3 g = ld3(dL + 3 * oidx) / div;
        ++paths;
        if (MODE == 0) path_nee_ds_bw(M, rng, x, w, M.ds_eps, g, tl, &sc->status);
        else if (MODE == 1) path_dt_bw(M, rng, x, w, M.ds_eps, g, tl, &sc->status);
        else if (MODE == 2) path_nee_drt_bw(M, rng, x, w, g, tl, &sc->status);
        else if (MODE == 3) path_nee_drtq_bw(M, rng, x, w, g, tl, &sc->status);
        else if (MODE == 4) path_nee_drtds_bw(M, rng, x, w, M.ds_eps, g, tl, &sc->status);
        else path_nee_sps_bw(M, rng, x, w, g, tl, &sc->status);
    }
    warp_add_counters(sc, paths, 0, tl);
}

// The reservoir branch of the DRT / DRTDS wavefront (vrt_wave_drt.cu) in three
// steps.  k_drt_branch_pre, one thread per path of the round: the primal left
// the reservoir vertex and the stream position at its end in resv (4 float4
// per path: vertex and its weight, direction and the running total -- 0 for a
// primary ray that missed the medium --, throughput, stream position); paths
// handed to the sequential form (first-collision word kSpilled) are skipped.
// It samples the branch position (_NEE_DRT.h:233-235; DS: the defensive
// collision position, no branch at weight 0) and its light rays, and appends
// an item: the nested path's start (position, direction, stream position, path
// id and stream word) and what the scatter needs (light terms, weights).  The
// nested scattered-only NEE paths run on the state machine
// (k_nee_fw<FW_BRANCH>); k_drt_branch_post adds their estimates and scatters
// at the branch position.
template <bool DS>
__global__ void __launch_bounds__(256) k_drt_branch_pre(DMedium M, PathSrc S, uint64_t n_paths, uint64_t p_begin,
                                                         const unsigned long long* next_path, uint64_t seed,
                                                         const float* __restrict__ info,
                                                         const float4* __restrict__ resv, float4* items,
                                                         float4* post, unsigned long long* n_items, DScratch* sc) {
    constexpr uint32_t kSpilledPath = 0xfffffffdu;  // the first-collision word of a handed-over path
    unsigned long long end = *next_path;
    if (end > n_paths) end = n_paths;
    const uint64_t n_round = end > p_begin ? end - p_begin : 0;
    Tally tl;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n_round;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const float4 r1 = resv[4 * k + 1];
        if (!(r1.w > 0.0f)) continue;  // the primary ray missed the medium: no branch
        if (__float_as_uint(info[8 * k + 7]) == kSpilledPath) continue;
        const float4 r0 = resv[4 * k], r2 = resv[4 * k + 2], r3 = resv[4 * k + 3];
        const uint64_t pid = p_begin + k;
        Rng rng;
        rng.init(seed, pid, 0);
        rng.seek(Rng::Pos{__float_as_uint(r3.x), __float_as_uint(r3.y)});
        const float3 res_x = make_float3(r0.x, r0.y, r0.z), res_w = make_float3(r1.x, r1.y, r1.z);
        float tMin, d;
        boundary(M, res_x, res_w, tMin, d);
        float s_t, weight_t;
        if (DS) sample_collision_position_ds(M, rng, res_x, res_w, d, M.ds_eps, s_t, weight_t, tl, &sc->status);
        else sample_transmittance_position(M, rng, res_x, res_w, d, s_t, weight_t, tl, &sc->status);
        if (DS && !(weight_t > 0.0f)) continue;
        const float3 xs = res_x + res_w * s_t;
        float3 ls_dir;
        const float3 Ls_env = environment_sample(M, rng, ls_dir);
        float3 Ls = transmittance(M, rng, xs, ls_dir, tl, &sc->status) * Ls_env * phase(M, res_w, ls_dir);
        if (M.has_sun)
            Ls = Ls + transmittance(M, rng, xs, M.sun_dir, tl, &sc->status) * M.sun_L * phase(M, res_w, M.sun_dir);
        const float3 ws = phase_sample(M, rng, res_w);
        const unsigned long long i = atomicAdd(n_items, 1ull);
        items[3 * i] = make_float4(xs.x, xs.y, xs.z, __uint_as_float(rng.n));
        items[3 * i + 1] = make_float4(ws.x, ws.y, ws.z, __uint_as_float(rng.ntr));
        items[3 * i + 2] = make_float4(__uint_as_float((uint32_t)pid), __uint_as_float((uint32_t)(pid >> 32)),
                                       __uint_as_float(0u), 0.0f);
        post[3 * i] = make_float4(Ls.x, Ls.y, Ls.z, weight_t);
        post[3 * i + 1] = make_float4(r2.x, r2.y, r2.z, r1.w);
        post[3 * i + 2] = make_float4(r0.w, 0.0f, 0.0f, 0.0f);
    }
    warp_add_counters(sc, 0, 0, tl);
}

// The DRTQ adjoint's scatter terms (_NEE_DRTQ.h:156-165, :249-259), one
// thread per segment: the round's segment 0s (the primal wrote them in resv,
// 3 float4 per path, length 0 for a primary ray that missed the medium) and
// the segments after scattering vertices (segs, *n_segs of them); segments of
// paths handed to the sequential form are skipped.  Each term draws from its
// segment's stream (Rng::segment_stream): the transmittance-sampled position,
// then in_scattering's light rays and direction; its nested scattered-only
// NEE path is appended as an item for k_nee_fw<FW_BRANCH> and
// k_drt_branch_post<2> scatters.
__global__ void __launch_bounds__(256) k_drtq_segment_pre(DMedium M, uint64_t n_paths, uint64_t p_begin,
                                                           const unsigned long long* next_path,
                                                           const unsigned long long* n_segs, uint64_t cap_segs,
                                                           uint64_t seed, const float* __restrict__ info,
                                                           const float4* __restrict__ resv,
                                                           const float4* __restrict__ segs, float4* items, float4* post,
                                                           unsigned long long* n_items, DScratch* sc) {
    constexpr uint32_t kSpilledPath = 0xfffffffdu;  // the first-collision word of a handed-over path
    unsigned long long end = *next_path;
    if (end > n_paths) end = n_paths;
    const uint64_t n_round = end > p_begin ? end - p_begin : 0;
    unsigned long long ns = *n_segs;
    if (ns > cap_segs) ns = cap_segs;
    Tally tl;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_round + ns;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4* g = i < n_round ? resv + 4 * i : segs + 3 * (i - n_round);
        const float4 a = g[0], b = g[1], c = g[2];
        if (i < n_round && !(a.w > 0.0f)) continue;  // the primary ray missed the medium
        const uint64_t k = __float_as_uint(c.w);     // the path's index in the round
        if (__float_as_uint(info[8 * k + 7]) == kSpilledPath) continue;
        const uint64_t pid = p_begin + k;
        Rng rng;
        rng.init(seed, pid, 0);
        rng = rng.segment_stream(__float_as_uint(b.w));
        const float3 x = make_float3(a.x, a.y, a.z), w = make_float3(b.x, b.y, b.z);
        float s_t, weight_t;
        sample_transmittance_position(M, rng, x, w, a.w, s_t, weight_t, tl, &sc->status);
        const float3 xs = x + w * s_t;
        float3 ls_dir;  // in_scattering (_NEE_DRTQ.h:45-55) up to its nested path
        const float3 Ls_env = environment_sample(M, rng, ls_dir);
        float3 Ls = transmittance(M, rng, xs, ls_dir, tl, &sc->status) * Ls_env * phase(M, w, ls_dir);
        if (M.has_sun) Ls = Ls + transmittance(M, rng, xs, M.sun_dir, tl, &sc->status) * M.sun_L * phase(M, w, M.sun_dir);
        const float3 ws = phase_sample(M, rng, w);
        const unsigned long long o = atomicAdd(n_items, 1ull);
        items[3 * o] = make_float4(xs.x, xs.y, xs.z, __uint_as_float(rng.n));
        items[3 * o + 1] = make_float4(ws.x, ws.y, ws.z, __uint_as_float(rng.ntr));
        items[3 * o + 2] = make_float4(__uint_as_float(rng.plo), __uint_as_float(rng.phi), __uint_as_float(rng.stream),
                                       __uint_as_float((uint32_t)k));
        post[3 * o] = make_float4(Ls.x, Ls.y, Ls.z, weight_t);
        post[3 * o + 1] = make_float4(c.x, c.y, c.z, 0.0f);
        post[3 * o + 2] = make_float4(__uint_as_float((uint32_t)pid), __uint_as_float((uint32_t)(pid >> 32)), 0.0f, 0.0f);
    }
    warp_add_counters(sc, 0, 0, tl);
}

// _NEE_DRT.h:261-268 (MODE 1, DRTDS: _NEE_DRTDS.h:248-251): the branch
// estimate (light terms + the nested path's) weighed by the reservoir and
// scattered at the branch position.  MODE 2, DRTQ (_NEE_DRTQ.h:52-54,
// :162-164): a segment's in-scattered light times W, MIS-weighted.
template <int MODE>
__global__ void __launch_bounds__(256) k_drt_branch_post(DMedium M, PathSrc S, uint64_t n_items,
                                                          const float4* __restrict__ items,
                                                          const float4* __restrict__ post, const float* __restrict__ R,
                                                          const float* dL, float div, DScratch* sc) {
    Tally tl;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_items;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float4 a = items[3 * i], c = MODE == 2 ? post[3 * i + 2] : items[3 * i + 2];
        const float4 p0 = post[3 * i], p1 = post[3 * i + 1], p2 = post[3 * i + 2];
        const uint64_t pid = (uint64_t)__float_as_uint(c.x) | ((uint64_t)__float_as_uint(c.y) << 32);
        const long long o = S.is_camera ? (long long)(pid % (uint64_t)S.npix) : (long long)pid;
        const float3 dL_dR = ld3(dL + 3 * o) / div;
        const float3 xs = make_float3(a.x, a.y, a.z);
        float3 Ls = make_float3(p0.x, p0.y, p0.z) + 1.0f * ld3(R + 3 * i);
        if (MODE == 2) {
            Ls = albedo(M, xs, tl) * Ls;
            const float sigma_t = sigma(M, xs, tl);
            const float mis_T = 1.0f / (1.0f + sigma_t * sigma_t);
            sigma_bw(M, xs, mis_T * p0.w * dot(dL_dR, make_float3(p1.x, p1.y, p1.z) * Ls), tl);
            continue;
        }
        Ls = Ls * make_float3(p1.x, p1.y, p1.z) * p0.w * albedo(M, xs, tl);
        const float total_weight = p1.w, res_P = p2.x;
        if (MODE == 1) {
            sigma_bw(M, xs, dot(dL_dR, Ls) * total_weight / res_P, tl);
        } else {
            const float sigma_xs = sigma(M, xs, tl);
            const float mis_T = 1.0f / (1.0f + sigma_xs * sigma_xs);
            sigma_bw(M, xs, dot(dL_dR, Ls) * mis_T * total_weight / res_P, tl);
        }
    }
    warp_add_counters(sc, 0, 0, tl);
}

// mode 0 DRT, 1 DRTDS (one branch per path of the round, from resv), 2 DRTQ
// (one scatter term per segment: the round's segment 0s in resv, then the
// *n_segs segments in segs)
int launch_drt_branch(const DMedium& M, int mode, const PathSrc& src, uint64_t n_paths, uint64_t p_begin,
                      const unsigned long long* next_path, uint64_t seed, const float* dL, float div, const float* info,
                      const float4* resv, uint64_t max_round, const float4* segs, const unsigned long long* n_segs,
                      uint64_t max_segs, float4* items, float4* post, float* R, unsigned long long* n_items,
                      DScratch* scratch, int num_sms, cudaStream_t stream) {
    if (max_round == 0) return 0;
    KernelScope ks(VRT_K_DRT_BRANCH, stream);
    // n_items[0]: the items appended, n_items[1]: the nested paths' work counter
    cudaError_t e = cudaMemsetAsync(n_items, 0, 2 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const uint64_t need = (max_round + (mode == 2 ? max_segs : 0) + 255) / 256;
    int blocks = (int)(need < (uint64_t)num_sms * 16 ? need : (uint64_t)num_sms * 16);
    if (mode == 2)
        k_drtq_segment_pre<<<blocks, 256, 0, stream>>>(M, n_paths, p_begin, next_path, n_segs, max_segs, seed, info,
                                                        resv, segs, items, post, n_items, scratch);
    else if (mode == 1)
        k_drt_branch_pre<true><<<blocks, 256, 0, stream>>>(M, src, n_paths, p_begin, next_path, seed, info, resv,
                                                             items, post, n_items, scratch);
    else
        k_drt_branch_pre<false><<<blocks, 256, 0, stream>>>(M, src, n_paths, p_begin, next_path, seed, info, resv,
                                                              items, post, n_items, scratch);
    unsigned long long n = 0;
    if ((e = cudaMemcpyAsync(&n, n_items, sizeof(n), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return launch_status(e);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
    int launches = 1;
    if (n) {  // the nested paths on the state machine, then the scatters
        CacheIO io = {};
        io.pR = R;
        io.branch = items;
        io.queue = n_items + 1;
        int pb = persistent_blocks((const void*)k_nee_fw<FW_BRANCH>, 256, num_sms);
        const uint64_t nb = (n + 255) / 256;
        if ((uint64_t)pb > nb) pb = (int)nb;
        k_nee_fw<FW_BRANCH><<<pb, 256, 0, stream>>>(M, src, n, seed, nullptr, 1.0f, scratch, io);
        const uint64_t np = (n + 255) / 256;
        blocks = (int)(np < (uint64_t)num_sms * 16 ? np : (uint64_t)num_sms * 16);
        if (mode == 2) k_drt_branch_post<2><<<blocks, 256, 0, stream>>>(M, src, n, items, post, R, dL, div, scratch);
        else if (mode == 1) k_drt_branch_post<1><<<blocks, 256, 0, stream>>>(M, src, n, items, post, R, dL, div, scratch);
        else k_drt_branch_post<0><<<blocks, 256, 0, stream>>>(M, src, n, items, post, R, dL, div, scratch);
        launches += 2;
    }
    count_launches(launches);
    return launch_status(cudaGetLastError());
}

// ------------------------------------------------------------------------
// Host launchers
// ------------------------------------------------------------------------
int launch_radiance_fw(const DMedium& M, int integrator, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       float* out, float scale, DScratch* scratch, int num_sms, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (integrator == 0) {
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        int blocks = persistent_blocks((const void*)k_nee_fw<FW_PLAIN>, 256, num_sms);
        uint64_t need = (n_paths + 255) / 256;
        if ((uint64_t)blocks > need) blocks = (int)need;
        CacheIO io = {};
        k_nee_fw<FW_PLAIN><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, scratch, io);
    } else {  // DT: the persistent state machine
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        int blocks = persistent_blocks((const void*)k_dt_fw_sm, 256, num_sms);
        const uint64_t nb = (n_paths + 255) / 256;
        if ((uint64_t)blocks > nb) blocks = (int)nb;
        k_dt_fw_sm<<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, scratch);
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_cache_paths(const DMedium& M, int mode, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                       float scale, const CacheIO& io, DScratch* scratch, int num_sms, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const void* kern = mode == FW_CUT ? (const void*)k_nee_fw<FW_CUT> : (const void*)k_nee_fw<FW_TRAIN>;
    int blocks = persistent_blocks(kern, 256, num_sms);
    uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)need;
    if (mode == FW_CUT) k_nee_fw<FW_CUT><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, scratch, io);
    else k_nee_fw<FW_TRAIN><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, scratch, io);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

// targets of the recorded collisions: (R_final - R_k) / W_k, R_final per path
__global__ void k_cache_targets(float* __restrict__ smp, const float* __restrict__ pR, long long n_paths, int rec) {
    const long long n = n_paths * rec;
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
        float* o = smp + 3 * r;
        const float3 Wk = ld3(o + 9 * n);
        if (Wk.x == 0.0f && Wk.y == 0.0f && Wk.z == 0.0f) continue;  // not reached: NaN target already
        const float3 num = ld3(pR + 3 * (r / rec)) - ld3(o + 6 * n);
        st3(o + 6 * n, make_float3(num.x / Wk.x, num.y / Wk.y, num.z / Wk.z));
    }
}

int launch_cache_targets(float* smp, const float* pR, long long n_paths, int rec, cudaStream_t stream) {
    const long long n = n_paths * rec;
    if (n == 0) return 0;
    long long b = (n + 255) / 256;
    k_cache_targets<<<(int)(b < 4096 ? b : 4096), 256, 0, stream>>>(smp, pR, n_paths, rec);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_radiance_bw(const DMedium& M, int bw_mode, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       const float* dL, float div, DScratch* scratch, int num_sms, cudaStream_t stream,
                       const unsigned long long* pids) {
    if (n_paths == 0) return 0;
    if (bw_mode == 0) return launch_nee_ds_bw(M, src, n_paths, seed, dL, div, scratch, num_sms, stream, pids);
    if (bw_mode == 1 && !pids) {  // DT: the persistent state machine
        cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        int blocks = persistent_blocks((const void*)k_dt_bw, 256, num_sms);
        const uint64_t nb = (n_paths + 255) / 256;
        if ((uint64_t)blocks > nb) blocks = (int)nb;
        k_dt_bw<<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch);
        count_launches(1);
        return launch_status(cudaGetLastError());
    }
    // DRTQ's segment streams carry the path id in 40 bits
    if (bw_mode == 3 && !pids && n_paths >= (1ull << 40)) return VRT_E_UNSUPPORTED;
    uint64_t need = (n_paths + 255) / 256;
    int blocks = (int)(need < (uint64_t)num_sms * 16 ? need : (uint64_t)num_sms * 16);
    if (bw_mode == 1) k_path_bw<1><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    else if (bw_mode == 2) k_path_bw<2><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    else if (bw_mode == 3) k_path_bw<3><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    else if (bw_mode == 4) k_path_bw<4><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    else k_path_bw<5><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
