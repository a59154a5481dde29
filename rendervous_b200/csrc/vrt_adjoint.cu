// vrt_adjoint.cu -- the NEE_DS path-replay adjoint as a persistent state machine (sm_100a).
//
// Restates include/vr_path_integrator_NEE_DS.h:6-206 (primal pass, then a replay
// that scatters dL/dsigma and dL/dalbedo) with the transmittance adjoints of
// include/vr_transmittance_RT.h:51-141 / _DT.h:30-90, exactly as
// path_nee_ds_bw in vrt_path.cu does one path per thread.  Here every lane owns
// one path and each loop iteration performs ONE free-flight step of whatever
// segment the lane is in:
//
//   PRIMARY  the path itself (primal pass, then the replay)
//   TRFW     a shadow ray's transmittance estimate (ratio or delta tracking)
//   TRBW1    first pass of a transmittance adjoint (its own estimate)
//   TRBW2    second pass of that adjoint, scattering dL/dsigma
//
// so the sigma gather and the gradient scatter are issued by the whole warp
// together.  Shadow rays draw from forks of the path's stream (fork j for the
// j-th transmittance of the path), so they can run after the path's own draws
// of a vertex (environment direction, phase direction) without changing any
// value: the result is draw-for-draw that of the sequential definition.
#include <cuda_runtime.h>

#include "vrt_device.cuh"
#include "vrt_internal.h"
#include "vrt_tracking.cuh"

namespace vrt {

namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kCap = 1 << 26;  // total steps of one path (VRT_E_ITER_CAP)

enum : int { S_DEAD = 0, S_PRIMARY = 1, S_TRFW = 2, S_TRBW1 = 3, S_TRBW2 = 4 };
enum : int { E_NONE = 0, E_COLLIDE = 1, E_END = 2, E_SEG_DONE = 3, E_SEG_ABORT = 4 };
enum : int { L_ENV = 0, L_SUN = 1 };

struct Lane {
    Flight ff;           // the current free flight (residual optical depth)
    Rng rng;             // active stream
    Rng::Pos ppos;       // the path stream, parked while a shadow stream runs
    uint4 pbuf;
    uint32_t pstream;
    // path
    float3 x0, w0;       // primary ray (the replay restarts from it)
    Rng::Pos pos0;       // path stream position after the camera draws
    float3 x, w, W, R, Rsp, dLdR;
    float d, null_W;
    int bounces;
    bool scattered, replay;
    long long oidx;
    uint32_t steps;
    // vertex
    float3 wnee, env, wo, acc;
    float ph_nee, ph_sun, T_nee, T_sun, dTnee, dTsun;
    float s_hit, m_hit, Pc_hit;
    uint32_t jfork;
    float bt0[2], bt1[2];  // shadow-ray box interval per light (tMax < tMin: miss)
    // segment
    int state, light;
    float3 sx;
    float sd, T, outT, dLdT;
};

__device__ __forceinline__ float3 shadow_dir(const DMedium& M, const Lane& L) {
    return L.light == L_ENV ? L.wnee : M.sun_dir;
}

__device__ __forceinline__ Rng fork_at(const Lane& L, uint32_t j) {
    Rng r;
    r.k0 = L.rng.k0; r.k1 = L.rng.k1; r.plo = L.rng.plo; r.phi = L.rng.phi;
    r.stream = L.pstream + 2u * (1u + j);
    r.n = 0; r.ntr = 0;
    return r;
}
__device__ __forceinline__ void park(Lane& L) {
    L.ppos = L.rng.pos();
    L.pbuf = L.rng.buf;
    L.pstream = L.rng.stream;
}
__device__ __forceinline__ void unpark(Lane& L) {
    L.rng.stream = L.pstream;
    L.rng.n = L.ppos.n;
    L.rng.ntr = L.ppos.ntr;
    L.rng.buf = L.pbuf;
}

// Starts a transmittance segment of kind `st` (TRFW / TRBW1 / TRBW2) for the
// current light from the vertex L.x.  Returns E_NONE when a tracking segment
// begins, E_SEG_DONE when it is already complete (missed boundary), or
// E_SEG_ABORT for a skipped adjoint (dL/dT == 0).
__device__ __forceinline__ int begin_segment(const DMedium& M, Lane& L, int st, Tally& tl, uint32_t* status) {
    const float3 dir = shadow_dir(M, L);
    const uint32_t j = L.jfork + (uint32_t)L.light;
    if (M.tr_mode >= 2) {  // DDA, GRT, GDT: evaluated inline
        if (st == S_TRFW) {
            if (M.tr_mode == 2) L.T = transmittance_dda<false>(M, L.x, dir, tl);
            else if (M.tr_mode == 3) L.T = transmittance_dda<true>(M, L.x, dir, tl);
            else {
                Rng r = fork_at(L, j);
                L.T = M.tr_mode == 4 ? transmittance_grid_tracking<false>(M, r, L.x, dir, tl, status)
                                     : transmittance_grid_tracking<true>(M, r, L.x, dir, tl, status);
            }
            return E_SEG_DONE;
        }
        if (M.tr_mode == 2) transmittance_dda_bw<false>(M, L.x, dir, L.dLdT, tl);
        else if (M.tr_mode == 3) transmittance_dda_bw<true>(M, L.x, dir, L.dLdT, tl);
        return E_SEG_ABORT;  // nothing more to run for this light (GRT / GDT have no backward)
    }
    if (st != S_TRFW && L.dLdT == 0.0f) return E_SEG_ABORT;  // _RT.h:53 / _DT.h:32
    // the vertex's box interval for this light, computed once per vertex
    const float tMin = L.light == L_ENV ? L.bt0[0] : L.bt0[1];
    const float tMax = L.light == L_ENV ? L.bt1[0] : L.bt1[1];
    if (!(tMax >= tMin)) {
        L.T = 1.0f;
        return st == S_TRFW ? E_SEG_DONE : E_SEG_ABORT;
    }
    if (L.state == S_PRIMARY) park(L);
    L.rng = fork_at(L, j);
    L.ff = Flight();
    L.sx = L.x + dir * tMin;
    L.sd = tMax - tMin;
    L.T = 1.0f;
    L.state = st;
    (void)status;
    return E_NONE;
}

// The transmittance maps' boundary test (vr_transmittance_RT.h:5-10) for both
// shadow directions of the current vertex; a miss is stored as tMax < tMin.
__device__ __forceinline__ void shadow_intervals(const DMedium& M, Lane& L) {
    float a, b;
    if (boundary(M, L.x, L.wnee, a, b)) { L.bt0[0] = a; L.bt1[0] = b; }
    else { L.bt0[0] = 1.0f; L.bt1[0] = 0.0f; }
    if (M.has_sun && boundary(M, L.x, M.sun_dir, a, b)) { L.bt0[1] = a; L.bt1[1] = b; }
    else { L.bt0[1] = 1.0f; L.bt1[1] = 0.0f; }
}

// After the path's own draws of a replayed vertex: decide what runs next.
// Sequence per light: TRFW env, TRFW sun, (R update), TRBW1/2 env, TRBW1/2 sun.
__device__ __forceinline__ void path_resume(Lane& L) {
    unpark(L);
    L.ff = Flight();
    L.state = S_PRIMARY;
}

}  // namespace

// pids: when not null, work item q is path pids[q] (the paths the NEE_DS
// wavefront handed over); else path q.
__global__ void __launch_bounds__(256, 2) k_nee_ds_bw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                    const float* __restrict__ dL, float div, DScratch* sc,
                                                    const unsigned long long* __restrict__ pids) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    Lane L;
    L.state = S_DEAD;
    bool exhausted = false;
    uint32_t n_paths_done = 0;
    Tally tl;

    while (true) {
        // ---- refill dead lanes (one atomic per warp)
        unsigned want = __ballot_sync(kAll, L.state == S_DEAD && !exhausted);
        if (want) {
            int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
            base = __shfl_sync(kAll, base, leader);
            if (L.state == S_DEAD && !exhausted) {
                uint64_t pid = base + __popc(want & ((1u << lane) - 1u));
                if (pid >= n_paths) {
                    exhausted = true;
                } else {
                    if (pids) pid = pids[pid];
                    L.rng.init(seed, pid, 0);
                    if (S.is_camera) {
                        long long p = (long long)(pid % (uint64_t)S.npix);
                        camera_pixel_ray(S.cam, p, L.rng, L.x0, L.w0, &sc->status);
                        L.oidx = p;
                    } else {
                        L.x0 = ld3(S.rays + 6 * pid);
                        L.w0 = ld3(S.rays + 6 * pid + 3);
                        L.oidx = (long long)pid;
                    }
                    L.dLdR = ld3(dL + 3 * L.oidx) / div;
                    L.pos0 = L.rng.pos();
                    L.pstream = L.rng.stream;
                    float tMin, tMax;
                    boundary(M, L.x0, L.w0, tMin, tMax);
                    L.x = L.x0 + L.w0 * tMin;
                    L.w = L.w0;
                    L.d = tMax - tMin;
                    L.W = f3(1.0f);
                    L.R = f3(0.0f);
                    L.Rsp = f3(0.0f);
                    L.null_W = 1.0f;
                    L.scattered = false;
                    L.replay = false;
                    L.bounces = 0;
                    L.steps = 0;
                    L.ff = Flight();
                    L.state = S_PRIMARY;
                    ++n_paths_done;
                }
            }
        }
        if (__all_sync(kAll, L.state == S_DEAD && exhausted)) break;
        if (L.state == S_DEAD) continue;

        int ev = E_NONE;
        if (L.state == S_PRIMARY && !(L.d > EPS)) {
            ev = E_END;  // the while (d > EPS) test of the primal / replay loop
        } else {
            // ---- one free flight of the current segment; majorant-brick faces
            // it crosses are handled in the inner loop without new draws
            const bool prim = L.state == S_PRIMARY;
            const float3 v = prim ? L.w : shadow_dir(M, L);
            if (L.ff.tau < 0.0f) ++tl.steps;
            L.ff.sample(L.rng);
            bool need = false;
            float m = 0.0f, t = 0.0f;
            for (int k = 0;; ++k) {
                if (k >= kStepCap) {
                    raise_status(&sc->status, 4);
                    L.steps = (uint32_t)kCap;  // retire the lane below
                    break;
                }
                float md;
                if (prim) {
                    // primal: + 2 eps + 0.1 (_NEE_DS.h:36); replay: the same, or the
                    // reference's x1.2 + 2 eps (_NEE_DS.h:120) under ds_compat
                    const float mj = L.ff.bk.query(M, L.x, v, md);
                    m = (L.replay && M.ds_compat) ? gmax(EPS, mj * 1.2f + 2.0f * eps) : gmax(EPS, mj + 2.0f * eps + 0.1f);
                    t = L.ff.tau / m;
                    L.x = L.x + v * gmin(t, md);
                    if (t > md) {
                        L.d -= md;
                        L.ff.cross(m, md);
                        L.ff.bk.advance(M);
                        if (!(L.d > EPS)) { ev = E_END; break; }
                        continue;
                    }
                    L.ff.used();
                    if (t > L.d) ev = E_END;
                    else need = true;
                    L.ff.bk.move(t);
                    break;
                }
                const float add = L.state == S_TRFW ? 0.0f : 0.1f;  // adjoint majorant +0.1 (_RT.h:75, _DT.h:48)
                m = gmax(0.0000001f, L.ff.bk.query(M, L.sx, v, md) + add);
                if (M.tr_mode == 0) {
                    t = L.ff.tau / m;
                    if (md < L.sd && t > md) {
                        L.sx = L.sx + v * md;
                        L.sd -= md;
                        L.ff.cross(m, md);
                        L.ff.bk.advance(M);
                        continue;
                    }
                    L.ff.used();
                    float dt = gmin(t, gmin(L.sd, md));
                    L.ff.bk.move(dt);
                    L.sx = L.sx + v * dt;
                    L.sd -= dt;
                    if (L.sd <= 0.0000001f) ev = E_SEG_DONE;
                    else need = true;
                    break;
                }
                float dt = L.ff.tau / m;
                float tt = gmin(md, dt);
                L.sx = L.sx + v * tt;
                L.sd -= tt;
                if (L.sd <= 0.0000001f) { L.ff.used(); ev = E_SEG_DONE; break; }
                if (dt > md) { L.ff.cross(m, md); L.ff.bk.advance(M); continue; }
                L.ff.used();
                L.ff.bk.move(tt);
                need = true;
                break;
            }
            float gsc = 0.0f;  // dL/dsigma to scatter at the looked-up point
            if (need) {
                const float s = sigma(M, prim ? L.x : L.sx, tl);
                if (prim) {
                    const float Pc = (s + eps) / m;
                    if (L.rng.uniform() >= Pc) {  // null collision
                        if (L.replay) gsc = dot(L.dLdR, -L.R / m / (1.0f - s / m));
                        L.W = L.W * ((1.0f - s / m) / (1.0f - Pc));
                        L.d -= t;
                    } else {
                        ev = E_COLLIDE;
                        L.s_hit = s;
                        L.m_hit = m;
                        L.Pc_hit = Pc;
                        if (L.replay) gsc = dot(L.dLdR, s < EPS ? L.Rsp / eps : L.R / s);
                    }
                } else if (M.tr_mode == 0) {
                    const float r = 1.0f - s / m;
                    L.T *= r;
                    if (L.state == S_TRBW2) gsc = -L.outT * L.dLdT / m / r;
                    const float thr = L.state == S_TRFW ? 0.01f : 0.1f;
                    if (L.T < thr) {
                        if (L.state == S_TRBW2) {
                            L.rng.advance();
                            L.T = 1.0f;
                        } else if (L.rng.uniform() < 1.0f - L.T) {
                            L.T = 0.0f;
                            ev = E_SEG_ABORT;
                        } else {
                            L.T = 1.0f;
                        }
                    }
                } else {
                    if (L.state == S_TRBW2) {
                        L.rng.advance();
                        gsc = -L.dLdT / m / (1.0f - s / m);
                    } else if (L.rng.uniform() < s / m) {
                        L.T = 0.0f;
                        ev = E_SEG_ABORT;
                    }
                }
            }
            if (gsc != 0.0f) sigma_bw(M, prim ? L.x : L.sx, gsc, tl);  // one scatter per iteration, warp-wide
            if (++L.steps > (uint32_t)kCap) {
                raise_status(&sc->status, 4);
                L.state = S_DEAD;
                continue;
            }
        }

        // ---- events (divergent, cheap)
        while (ev != E_NONE) {
            if (L.state == S_PRIMARY && (ev == E_COLLIDE || ev == E_END)) {
                if (ev == E_COLLIDE && !L.replay) {
                    // primal vertex (_NEE_DS.h:48-99)
                    L.scattered = true;
                    const float s = L.s_hit;
                    if (s < EPS) {
                        if (L.null_W < EPS) { L.W = f3(0.0f); ev = E_END; continue; }
                        L.null_W = 0.0f;
                    } else {
                        L.W = L.W * ((s / L.m_hit) / L.Pc_hit);
                    }
                    const float3 sa = albedo(M, L.x, tl);
                    L.acc = L.W * (f3(1.0f) - sa) * M.emission;
                    L.W = L.W * sa;
                    L.env = environment_sample(M, L.rng, L.wnee);
                    L.ph_nee = phase(M, L.w, L.wnee);
                    L.ph_sun = M.has_sun ? phase(M, L.w, M.sun_dir) : 0.0f;
                    shadow_intervals(M, L);
                    L.jfork = L.rng.ntr;
                    L.rng.ntr += M.has_sun ? 2u : 1u;
                    const bool capped = M.max_bounces > 0 && L.bounces + 1 >= M.max_bounces;
                    if (!capped) L.wo = phase_sample(M, L.rng, L.w);
                    L.light = L_ENV;
                    ev = begin_segment(M, L, S_TRFW, tl, &sc->status);
                } else if (ev == E_COLLIDE) {
                    // replayed vertex (_NEE_DS.h:151-203)
                    const float s = L.s_hit;
                    L.W = L.W * (s / L.m_hit / L.Pc_hit);
                    if (s < EPS) { ev = E_END; L.d = 0.0f; continue; }
                    const float3 sa = albedo(M, L.x, tl);
                    float3 dL_dsa = L.dLdR * L.W * -1.0f * M.emission;
                    L.R = L.R - L.W * (f3(1.0f) - sa) * M.emission;
                    dL_dsa = dL_dsa + L.dLdR * L.R / make_float3(gmax(EPS, sa.x), gmax(EPS, sa.y), gmax(EPS, sa.z));
                    albedo_bw(M, L.x, dL_dsa, tl);
                    L.env = environment_sample(M, L.rng, L.wnee);
                    L.ph_nee = phase(M, L.w, L.wnee);
                    L.ph_sun = M.has_sun ? phase(M, L.w, M.sun_dir) : 0.0f;
                    shadow_intervals(M, L);
                    L.jfork = L.rng.ntr;
                    L.rng.ntr += M.has_sun ? 2u : 1u;
                    L.wo = phase_sample(M, L.rng, L.w);
                    L.W = L.W * sa;
                    L.light = L_ENV;
                    ev = begin_segment(M, L, S_TRFW, tl, &sc->status);
                } else if (ev == E_END && !L.replay) {
                    // end of the primal pass (_NEE_DS.h:106-121): restart for the replay
                    if (!L.scattered) L.R = L.R + env_radiance(M, L.w) * L.W;
                    L.replay = true;
                    L.ff = Flight();
                    L.rng.seek(L.pos0);
                    L.W = f3(1.0f);
                    L.bounces = 0;
                    float tMin, tMax;
                    boundary(M, L.x0, L.w0, tMin, tMax);
                    L.x = L.x0 + L.w0 * tMin;
                    L.w = L.w0;
                    L.d = tMax - tMin;
                    ev = E_NONE;
                } else {  // E_END of the replay: the path is done
                    L.state = S_DEAD;
                    ev = E_NONE;
                }
                continue;
            }
            // ---- a transmittance segment ended (the lane is parked, or DDA inline)
            const int st = L.state;
            if (ev == E_SEG_DONE && st == S_TRBW1) {  // pass 1 complete: replay it with gradients
                L.outT = L.T;
                ev = begin_segment(M, L, S_TRBW2, tl, &sc->status);
                continue;
            }
            const bool was_fw = st == S_TRFW || (st == S_PRIMARY && ev == E_SEG_DONE);
            if (st != S_PRIMARY) path_resume(L);
            if (was_fw) {
                if (L.light == L_ENV) L.T_nee = L.T;
                else L.T_sun = L.T;
                if (L.light == L_ENV && M.has_sun) {
                    L.light = L_SUN;
                    ev = begin_segment(M, L, S_TRFW, tl, &sc->status);
                    continue;
                }
                if (!L.replay) {
                    // primal: accumulate this vertex's light and continue (_NEE_DS.h:86-99)
                    float3 added = L.acc + L.W * L.T_nee * L.env * L.ph_nee;
                    if (M.has_sun) added = added + L.W * L.T_sun * M.sun_L * L.ph_sun;
                    if (L.null_W < EPS) L.Rsp = L.Rsp + added;
                    else L.R = L.R + added;
                    if (M.max_bounces > 0 && ++L.bounces >= M.max_bounces) { L.W = f3(0.0f); ev = E_END; continue; }
                    if (all_less(L.W, EPS)) { L.W = f3(0.0f); ev = E_END; continue; }
                    L.w = L.wo;
                    float tMin;
                    boundary(M, L.x, L.w, tMin, L.d);
                    L.ff = Flight();
                    ev = E_NONE;
                    continue;
                }
                // replay: subtract this vertex's light, then run the transmittance adjoints
                L.dTnee = dot(L.dLdR, L.W * L.env * L.ph_nee);
                L.R = L.R - L.W * L.T_nee * L.env * L.ph_nee;
                if (M.has_sun) {
                    L.dTsun = dot(L.dLdR, L.W * M.sun_L * L.ph_sun);
                    L.R = L.R - L.W * L.T_sun * M.sun_L * L.ph_sun;
                }
                L.light = L_ENV;
                L.dLdT = L.dTnee;
                ev = begin_segment(M, L, S_TRBW1, tl, &sc->status);
                continue;
            }
            // an adjoint finished (pass 2 done, aborted in pass 1, or skipped)
            if (L.light == L_ENV && M.has_sun) {
                L.light = L_SUN;
                L.dLdT = L.dTsun;
                ev = begin_segment(M, L, S_TRBW1, tl, &sc->status);
                continue;
            }
            // the replayed vertex is complete (_NEE_DS.h:195-203)
            if (M.max_bounces > 0 && ++L.bounces >= M.max_bounces) { ev = E_END; L.d = 0.0f; continue; }
            if (all_less(L.W, EPS)) { ev = E_END; L.d = 0.0f; continue; }
            L.w = L.wo;
            float tMin;
            boundary(M, L.x, L.w, tMin, L.d);
            L.ff = Flight();
            ev = E_NONE;
        }
    }
    // per-warp counter flush
    unsigned long long pc = n_paths_done, s = tl.steps, l = tl.lookups, r = tl.reds, a = tl.albedo;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        pc += __shfl_down_sync(kAll, pc, o);
        s += __shfl_down_sync(kAll, s, o);
        l += __shfl_down_sync(kAll, l, o);
        r += __shfl_down_sync(kAll, r, o);
        a += __shfl_down_sync(kAll, a, o);
    }
    if (lane == 0) {
        atomicAdd(&sc->paths, pc);
        atomicAdd(&sc->steps, s);
        atomicAdd(&sc->lookups, l);
        atomicAdd(&sc->reds, r);
        atomicAdd(&sc->albedo, a);
    }
}

int launch_nee_ds_bw(const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, const float* dL, float div,
                     DScratch* scratch, int num_sms, cudaStream_t stream, const unsigned long long* pids) {
    cudaError_t e = cudaMemsetAsync(&scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    int blocks = persistent_blocks((const void*)k_nee_ds_bw, 256, num_sms);
    uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)need;
    k_nee_ds_bw<<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, scratch, pids);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
