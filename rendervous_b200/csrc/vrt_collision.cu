// vrt_collision.cu -- collision sampling and collision integrators (sm_100a).
//
//   DeltatrackingCollisionSampler  include/vr_collision_sampler_DT.h:1-134
//                                  (map form include/maps/collision_sampler_dt.h)
//   MCCollisionIntegrator          include/maps/collision_integrator_mc.h:1-41
//   GridDDACollisionIntegrator     include/vr_collision_integrator_DDA.h:1-207
//   exitance radiance              the emission, MCScatteredRadiance or
//                                  MCScatteredEmittedRadiance
//                                  (include/maps/scattered_radiance_mc.h,
//                                  scattered_emitted_radiance_mc.h) over
//                                  radiance = transmittance x environment
//
// MC: one path per thread, grid-stride (one tracking walk and one exitance per
// path).  DDA: persistent lanes refilled path by path, one cell (and its
// exitance) per iteration, so misses and short walks do not hold a warp.  A path's draws come from streams of
// its own Philox key: the collision sampler on stream 2, its adjoint on stream
// 4, exitance evaluation k on stream (k + 1) << 16 (its transmittance on the
// fork after it), the DDA's per-cell points on the path stream after the
// camera's draws.  The backward passes re-create those streams, so the
// adjoints differentiate the forward's own samples (the reference draws fresh
// seeds for every backward call).
//
// Compiled with -fmad=false, like the oracle's restatement, so a tracking
// decision is not flipped by a contracted multiply-add.
#include <cuda_runtime.h>

#include "../../include/vrt.h"
#include "vrt_internal.h"
#include "vrt_tracking.cuh"
#include "vrt_wave.cuh"

namespace vrt {
namespace {

using wave::out_index;
using wave::start_ray;

__device__ __forceinline__ Rng with_stream(const Rng& r, uint32_t s) {
    Rng o = r;
    o.stream = s;
    o.n = 0;
    o.ntr = 0;
    return o;
}
__device__ __forceinline__ uint32_t exitance_stream(long long k) { return (uint32_t)((k + 1) & 0x7fff) << 16; }

// include/vr_collision_sampler_DT.h:6-43.  Returns C (1 at a collision, else
// 0); out_t is the distance from x, out_T = 1 - C.  The free flight carries its
// residual optical depth across majorant-brick faces.
__device__ float collision_sample_dt(const DMedium& M, Rng& rng, float3 x, float3 w, float& out_t, float& out_T,
                                     Tally& tl, uint32_t* status) {
    out_T = 1.0f;
    out_t = 0.0f;
    float C = 0.0f;
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return C;
    const float d = tMax - tMin;
    x = x + w * tMin;
    float t = 0.0f;
    Flight ff;
    for (int it = 0;; ++it) {
        if (it >= kStepCap) {
            raise_status(status, 4);
            break;
        }
        float md;
        const float maj = ff.bk.query(M, x, w, md);
        if (ff.tau < 0.0f) ++tl.steps;
        const float tau = ff.sample(rng);
        const bool crosses = tau > md * maj;
        float dt = crosses ? md : tau / maj;
        dt = gmin(dt, d);
        x = x + w * dt;
        t += dt;
        if (t >= d - 0.0000001f) break;
        if (crosses) {
            ff.cross(maj, md);
            ff.bk.advance(M);
            continue;
        }
        ff.used();
        ff.bk.move(dt);
        if (rng.uniform() < sigma(M, x, tl) / maj) {
            out_T = 0.0f;
            C = 1.0f;
            break;
        }
    }
    out_t = tMin + t;
    return C;
}

// include/vr_collision_sampler_DT.h:45-134: the defensively sampled walk
// (majorant + 2 eps, Pc = (sigma + eps) / majorant) for the estimate, then the
// same draws again, scattering dL/dsigma at its collisions.
__device__ void collision_sample_dt_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float eps, float dL_dC,
                                       float dL_dT, Tally& tl, uint32_t* status) {
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return;
    const Rng before = rng;
    float out_T = 1.0f, C = 0.0f, s_t = 0.0f;
    const float d = tMax - tMin;
    x = x + w * tMin;
    const float3 ini_x = x;
    for (int pass = 0; pass < 2; ++pass) {
        float t = 0.0f;
        Flight ff;
        for (int it = 0;; ++it) {
            if (it >= kStepCap) {
                raise_status(status, 4);
                return;
            }
            float md;
            const float maj = gmax(0.0000000001f, ff.bk.query(M, x, w, md) + 2.0f * eps);
            const float tau = ff.sample(rng);
            const bool crosses = tau > md * maj;
            float dt = crosses ? md : tau / maj;
            dt = gmin(dt, d);
            x = x + w * dt;
            t += dt;
            if (t >= d - 0.0000001f) break;
            if (crosses) {
                ff.cross(maj, md);
                ff.bk.advance(M);
                continue;
            }
            ff.used();
            ff.bk.move(dt);
            const float s = sigma(M, x, tl);
            const float Pc = (s + eps) / maj;
            const bool hit = rng.uniform() < Pc;
            if (pass == 0) {
                if (hit) {
                    out_T = 0.0f;
                    C = 1.0f;
                    s_t = s / maj / Pc;
                    break;
                }
                out_T *= (1.0f - s / maj) / (1.0f - Pc);
            } else if (hit) {
                sigma_bw(M, x, dL_dC * (C / Pc) * (1.0f / maj), tl);
                break;
            } else {
                const float g = (dL_dT * out_T + dL_dC * C * s_t) / ((1.0f - s / maj) / (1.0f - Pc)) / (1.0f - Pc);
                sigma_bw(M, x, g * (-1.0f / maj), tl);
            }
        }
        rng = before;
        x = ini_x;
    }
}

// Exitance radiance at x towards wout (= -ray direction) by M.exitance_mode:
// 0 the emission; 1 sa(x) * rho * T(x, wo) * environment with (rho, wo) from
// the phase sampler at -wout (rho = 1 for the HG samplers); 2 the same plus
// (1 - sa) * emission.  rng is the evaluation's own stream.
__device__ float3 exitance(const DMedium& M, Rng& rng, float3 x, float3 wout, Tally& tl, uint32_t* status) {
    if (M.exitance_mode == 0) return emission_at(M, x);
    const float3 wo = phase_sample(M, rng, -wout);
    const float3 sa = albedo(M, x, tl);
    const float3 rad = env_radiance(M, wo) * transmittance(M, rng, x, wo, tl, status);
    float3 R = sa * 1.0f * rad;
    if (M.exitance_mode == 2) R = R + (f3(1.0f) - sa) * emission_at(M, x);
    return R;
}
// exitance() and its adjoint at one point on the same draws: the value
// (returned) and the adjoint of that value for dL, the phase sample, albedo and
// transmittance evaluated once.  Each factor gets the adjoint of the forward's
// expression (the reference's scattered maps hand (w, dL/dR) to the radiance
// map's backward and drop the dL/dR factor of the emission term of dL/dsa).
__device__ float3 exitance_fw_bw(const DMedium& M, const Rng& stream, float3 x, float3 wout, float3 dL, Tally& tl,
                                 uint32_t* status) {
    if (M.exitance_mode == 0) {
        emission_bw(M, x, dL, tl);
        return emission_at(M, x);
    }
    Rng rng = stream;
    const float3 wo = phase_sample(M, rng, -wout);
    const float3 sa = albedo(M, x, tl);
    Rng tr_rng = rng;
    const float Tr = transmittance(M, rng, x, wo, tl, status);
    const float3 env = env_radiance(M, wo);
    const float3 rad = env * Tr;
    float3 R = sa * 1.0f * rad;
    float3 dL_dsa = dL * rad * 1.0f;
    const float3 dL_drad = dL * sa * 1.0f;
    if (M.exitance_mode == 2) {
        const float3 em = emission_at(M, x);
        R = R + (f3(1.0f) - sa) * em;
        dL_dsa = dL_dsa - dL * em;
        emission_bw(M, x, dL * (f3(1.0f) - sa), tl);
    }
    albedo_bw(M, x, dL_dsa, tl);
    transmittance_bw(M, tr_rng, x, wo, dot(dL_drad, env), tl, status);
    return R;
}

// include/maps/collision_integrator_mc.h:8-18
__device__ float3 collision_integrate_mc(const DMedium& M, const Rng& rng, float3 x, float3 w, uint32_t& verts,
                                         Tally& tl, uint32_t* status) {
    Rng cs = with_stream(rng, 2);
    float t, Tt;
    const float C = collision_sample_dt(M, cs, x, w, t, Tt, tl, status);
    float3 eR = f3(0.0f);
    if (C != 0.0f) {
        ++verts;
        Rng xr = with_stream(rng, exitance_stream(0));
        eR = exitance(M, xr, w * t + x, -w, tl, status);
    }
    return eR * C + env_radiance(M, w) * Tt;
}
// include/maps/collision_integrator_mc.h:20-41: the forward's collision (same
// stream), the sampler's adjoint on its own stream, the exitance's adjoint on
// the forward's exitance draws.
__device__ void collision_integrate_mc_bw(const DMedium& M, const Rng& rng, float3 x, float3 w, float3 dL, Tally& tl,
                                          uint32_t* status) {
    Rng cs = with_stream(rng, 2);
    float t, Tt;
    const float C = collision_sample_dt(M, cs, x, w, t, Tt, tl, status);
    const float3 xt = w * t + x;
    float3 eR = f3(0.0f);
    if (C != 0.0f) eR = exitance_fw_bw(M, with_stream(rng, exitance_stream(0)), xt, -w, dL * C, tl, status);
    Rng cb = with_stream(rng, 4);
    collision_sample_dt_bw(M, cb, x, w, M.ds_eps, dot(dL, eR), dot(dL, env_radiance(M, w)), tl, status);
}

// dL/dsigma of a DDA cell, g, scattered into its 8 corners at the sample point a
__device__ __forceinline__ void dda_cell_scatter(const DMedium& M, const DDA& q, float3 a, float g, Tally& tl) {
    if (g == 0.0f || !M.sigma.grad) return;
    const float bx = 1.0f - a.x, by = 1.0f - a.y, bz = 1.0f - a.z;
    const float wt[8] = {g * bx * by * bz, g * a.x * by * bz, g * bx * a.y * bz, g * a.x * a.y * bz,
                         g * bx * by * a.z, g * a.x * by * a.z, g * bx * a.y * a.z, g * a.x * a.y * a.z};
#pragma unroll
    for (int c = 0; c < 8; ++c)
        red_add(M.sigma.grad + q.node(M.sigma, q.cx + (c & 1), q.cy + ((c >> 1) & 1), q.cz + (c >> 2)), wt[c]);
    tl.reds += 8;
}

// One cell of the DDA collision integrator (vr_collision_integrator_DDA.h:1-82):
// a random point of the cell (the path stream), the homogeneous transmittance
// exp(-dt sigma(point)) and the exitance there (stream exitance_stream(k)).
__device__ __forceinline__ void dda_collision_cell(const DMedium& M, DDA& q, Rng& rng, float3 w, long long k, float& Tr,
                                                   float& ct, float3& R, Tally& tl, uint32_t* status) {
    const float nt = gmin(q.d, gmin(q.alpha.x, gmin(q.alpha.y, q.alpha.z)));
    const float cell_t = mixf(ct, nt, rng.uniform());
    const float sv = q.interp(q.ialpha(cell_t));
    const float vt = expf(-(nt - ct) * sv);
    Rng xr = with_stream(rng, exitance_stream(k));
    const float3 Le = exitance(M, xr, q.x + w * cell_t, -w, tl, status);
    R = R + Le * (Tr * (1.0f - vt));
    Tr *= vt;
    ++tl.steps;
    ++tl.lookups;
    ct = nt;
    const int axis = q.advance_cell();
    q.shift_load(M.sigma, axis);
}

// include/vr_collision_integrator_DDA.h:85-207: the reference walks the cells
// twice -- for fw_T and the emitted total R, then again from the same cell
// draws scattering dL/dsigma = dL/dR . (T Le - fw_T env - R_rest) dt into the
// cell's corners and the exitance's adjoint dL/dR T (1 - v) at each point.
// With R_rest = R - P (P: the emitted part up to and including the cell) the
// scatter splits into dL/dR . (T Le + P) dt, known on the first walk, and
// -dL/dR . (fw_T env + R) dt, whose factor is known only at its end: so the
// first walk (dda_collision_bw_cell) evaluates each exitance once with its
// adjoint and scatters the first part, and a second walk over the same cells
// and draws -- without the exitances' light rays or corner loads -- scatters
// the second (dda_collision_g_cell).
__device__ __forceinline__ void dda_collision_bw_cell(const DMedium& M, DDA& q, Rng& rng, float3 w, float3 dL,
                                                      long long k, float& Tr, float& ct, float3& P, Tally& tl,
                                                      uint32_t* status) {
    const float nt = gmin(q.d, gmin(q.alpha.x, gmin(q.alpha.y, q.alpha.z)));
    const float cell_t = mixf(ct, nt, rng.uniform());
    const float3 a = q.ialpha(cell_t);
    const float sv = q.interp(a);
    const float dt = nt - ct;
    const float vt = expf(-dt * sv);
    const float3 Le = exitance_fw_bw(M, with_stream(rng, exitance_stream(k)), q.x + w * cell_t, -w,
                                     dL * (Tr * (1.0f - vt)), tl, status);
    P = P + Le * (Tr * (1.0f - vt));
    Tr *= vt;
    dda_cell_scatter(M, q, a, dot(dL, (Le * Tr + P) * dt), tl);
    ct = nt;
    const int axis = q.advance_cell();
    q.shift_load(M.sigma, axis);
}
__device__ __forceinline__ void dda_collision_g_cell(const DMedium& M, DDA& q, Rng& rng, float G, float& ct,
                                                     Tally& tl) {
    const float nt = gmin(q.d, gmin(q.alpha.x, gmin(q.alpha.y, q.alpha.z)));
    const float cell_t = mixf(ct, nt, rng.uniform());
    dda_cell_scatter(M, q, q.ialpha(cell_t), -G * (nt - ct), tl);
    ct = nt;
    q.advance_cell();
}

// A lane's next path from the scratch's work counter (one atomic per warp
// refill); all lanes call it together.
__device__ __forceinline__ bool take_path(DScratch* sc, bool want_path, uint64_t& p) {
    const unsigned want = __ballot_sync(0xffffffffu, want_path);
    if (!want) return false;
    const unsigned lane = threadIdx.x & 31u;
    const int leader = __ffs(want) - 1;
    unsigned long long base = 0;
    if ((int)lane == leader) base = atomicAdd(&sc->next_path, (unsigned long long)__popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!want_path) return false;
    p = base + __popc(want & ((1u << lane) - 1u));
    return true;
}

__device__ __forceinline__ void write_radiance(const PathSrc& S, float* out, float scale, uint64_t pid, float3 R) {
    const long long o = out_index(S, pid);
    if (S.is_camera) {
        atomicAdd(out + 3 * o + 0, R.x * scale);
        atomicAdd(out + 3 * o + 1, R.y * scale);
        atomicAdd(out + 3 * o + 2, R.z * scale);
    } else {
        out[3 * o + 0] = R.x;
        out[3 * o + 1] = R.y;
        out[3 * o + 2] = R.z;
    }
}

// per-warp sums of the lanes' counts into the context counters
__device__ __forceinline__ void collision_tally(DScratch* sc, uint32_t paths, uint32_t verts, const Tally& tl) {
    unsigned long long p = paths, v = verts, s = tl.steps, l = tl.lookups, r = tl.reds, a = tl.albedo;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        p += __shfl_down_sync(0xffffffffu, p, o);
        v += __shfl_down_sync(0xffffffffu, v, o);
        s += __shfl_down_sync(0xffffffffu, s, o);
        l += __shfl_down_sync(0xffffffffu, l, o);
        r += __shfl_down_sync(0xffffffffu, r, o);
        a += __shfl_down_sync(0xffffffffu, a, o);
    }
    if ((threadIdx.x & 31u) == 0u) {
        if (p) atomicAdd(&sc->paths, p);
        if (v) atomicAdd(&sc->vertices, v);
        if (s) atomicAdd(&sc->steps, s);
        if (l) atomicAdd(&sc->lookups, l);
        if (r) atomicAdd(&sc->reds, r);
        if (a) atomicAdd(&sc->albedo, a);
    }
}

// MC collision integrator, one path per thread, grid-stride
__global__ void __launch_bounds__(256) k_collision_mc_fw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                      float* __restrict__ out, float scale, DScratch* sc) {
    uint32_t paths = 0, verts = 0;
    Tally tl;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // the loop runs the same number of rounds in every lane of a warp, so the
    // warp-wide tally after it sees all 32 lanes
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_paths; base += stride) {
        const uint64_t pid = base + threadIdx.x;
        if (pid >= n_paths) continue;
        Rng rng;
        rng.init(seed, pid, 0);
        float3 x0, w0;
        start_ray(S, pid, rng, x0, w0, sc);
        const float3 R = collision_integrate_mc(M, rng, x0, w0, verts, tl, &sc->status);
        ++paths;
        write_radiance(S, out, scale, pid, R);
    }
    collision_tally(sc, paths, verts, tl);
}

__global__ void __launch_bounds__(256) k_collision_mc_bw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                      const float* __restrict__ dL, float div, DScratch* sc) {
    Tally tl;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_paths; base += stride) {
        const uint64_t pid = base + threadIdx.x;
        if (pid >= n_paths) continue;
        Rng rng;
        rng.init(seed, pid, 0);
        float3 x0, w0;
        start_ray(S, pid, rng, x0, w0, sc);
        const float3 d = ld3(dL + 3 * out_index(S, pid)) / div;
        collision_integrate_mc_bw(M, rng, x0, w0, d, tl, &sc->status);
    }
    collision_tally(sc, 0, 0, tl);
}

// The DDA collision integrator on persistent lanes: a lane takes the next
// path as soon as its walk ends, one cell (random point, transmittance,
// exitance and its light ray) per iteration, so misses and short walks do not
// wait for the warp's longest.  A path's draws and arithmetic are those of the
// per-path walk, cell for cell.
__global__ void __launch_bounds__(256) k_collision_dda_fw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                          float* __restrict__ out, float scale, DScratch* sc) {
    DDA q;
    Rng rng;
    float3 w = f3(0.0f), R = f3(0.0f);
    float Tr = 1.0f, ct = 0.0f;
    long long k = 0;
    uint64_t pid = 0;
    bool busy = false, exhausted = false;
    uint32_t paths = 0;
    Tally tl;
    while (true) {
        uint64_t p;
        if (take_path(sc, !busy && !exhausted, p)) {
            if (p >= n_paths) {
                exhausted = true;
            } else {
                pid = p;
                rng.init(seed, pid, 0);
                float3 x0;
                start_ray(S, pid, rng, x0, w, sc);
                ++paths;
                if (!q.init(M, x0, w)) {
                    write_radiance(S, out, scale, pid, env_radiance(M, w));
                } else {
                    q.load_all(M.sigma);
                    Tr = 1.0f;
                    ct = 0.0f;
                    R = f3(0.0f);
                    k = 0;
                    busy = true;
                }
            }
        }
        if (__all_sync(0xffffffffu, !busy && exhausted)) break;
        if (busy) {
            if (ct < q.d - 0.0001f && k < kStepCap) {
                dda_collision_cell(M, q, rng, w, k, Tr, ct, R, tl, &sc->status);
                ++k;
            } else {
                if (ct < q.d - 0.0001f) raise_status(&sc->status, 4);
                write_radiance(S, out, scale, pid, R + env_radiance(M, w) * Tr);
                busy = false;
            }
        }
    }
    collision_tally(sc, paths, 0, tl);
}

// Its adjoint: phase 0 the first walk (exitances and their adjoints), phase 1
// the second (the total-scaled part of the sigma scatter), from the stream
// position the first started at.
__global__ void __launch_bounds__(256) k_collision_dda_bw(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                          const float* __restrict__ dL, float div, DScratch* sc) {
    DDA q;
    Rng rng;
    Rng::Pos before = {0u, 0u};
    float3 w = f3(0.0f), g = f3(0.0f), P = f3(0.0f);
    float Tr = 1.0f, ct = 0.0f, G = 0.0f;
    long long k = 0;
    int phase = 0;
    bool busy = false, exhausted = false;
    Tally tl;
    while (true) {
        uint64_t p;
        if (take_path(sc, !busy && !exhausted, p)) {
            if (p >= n_paths) {
                exhausted = true;
            } else {
                rng.init(seed, p, 0);
                float3 x0;
                start_ray(S, p, rng, x0, w, sc);
                g = ld3(dL + 3 * out_index(S, p)) / div;
                if (!(g.x == 0.0f && g.y == 0.0f && g.z == 0.0f) && q.init(M, x0, w)) {
                    before = rng.pos();
                    q.load_all(M.sigma);
                    Tr = 1.0f;
                    ct = 0.0f;
                    P = f3(0.0f);
                    k = 0;
                    phase = 0;
                    busy = true;
                }
            }
        }
        if (__all_sync(0xffffffffu, !busy && exhausted)) break;
        if (busy) {
            if (phase == 0) {
                if (ct < q.d - 0.0001f) {
                    if (k >= kStepCap) {
                        raise_status(&sc->status, 4);
                        busy = false;
                    } else {
                        dda_collision_bw_cell(M, q, rng, w, g, k, Tr, ct, P, tl, &sc->status);
                        ++k;
                    }
                } else {
                    G = dot(g, env_radiance(M, w) * Tr + P);  // fw_T env + R
                    if (G == 0.0f || !M.sigma.grad) {
                        busy = false;
                    } else {
                        rng.seek(before);
                        q.reset(M);  // (the second walk reads no corner values: no loads)
                        ct = 0.0f;
                        phase = 1;
                    }
                }
            } else if (ct < q.d - 0.0001f) {
                dda_collision_g_cell(M, q, rng, G, ct, tl);
            } else {
                busy = false;
            }
        }
    }
    collision_tally(sc, 0, 0, tl);
}

// DeltatrackingCollisionSampler on rays: ray i draws from stream 2 of path i
// (its adjoint from stream 4), as inside the MC collision integrator.
__global__ void __launch_bounds__(256) k_collision_sample_fw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                             uint64_t seed, float* __restrict__ out3, DScratch* sc) {
    uint32_t paths = 0, verts = 0;
    Tally tl;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        if (i >= n) continue;
        Rng rng;
        rng.init(seed, (uint64_t)i, 2);
        float t, Tt;
        const float C = collision_sample_dt(M, rng, ld3(rays + 6 * i), ld3(rays + 6 * i + 3), t, Tt, tl, &sc->status);
        out3[3 * i] = C;
        out3[3 * i + 1] = t;
        out3[3 * i + 2] = Tt;
        ++paths;
        if (C != 0.0f) ++verts;
    }
    collision_tally(sc, paths, verts, tl);
}

__global__ void __launch_bounds__(256) k_collision_sample_bw(DMedium M, const float* __restrict__ rays, int64_t n,
                                                             uint64_t seed, const float* __restrict__ dL3,
                                                             DScratch* sc) {
    Tally tl;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        if (i >= n) continue;
        Rng rng;
        rng.init(seed, (uint64_t)i, 4);
        collision_sample_dt_bw(M, rng, ld3(rays + 6 * i), ld3(rays + 6 * i + 3), M.ds_eps, dL3[3 * i], dL3[3 * i + 2],
                               tl, &sc->status);
    }
    collision_tally(sc, 0, 0, tl);
}

int grid_blocks(uint64_t n, int num_sms) {
    uint64_t b = (n + 255) / 256;
    const uint64_t cap = (uint64_t)num_sms * 16;  // grid-stride beyond 16 blocks per SM
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// persistent grid of the lane kernels, at most one lane per path
int lane_blocks(const void* kernel, uint64_t n, int num_sms) {
    int b = persistent_blocks(kernel, 256, num_sms);
    const uint64_t need = (n + 255) / 256;
    if ((uint64_t)b > need) b = (int)need;
    return b < 1 ? 1 : b;
}

}  // namespace

int launch_collision_fw(const DMedium& M, int integrator, const PathSrc& S, uint64_t n_paths, uint64_t seed,
                        float* out, float scale, DScratch* sc, int num_sms, cudaStream_t stream) {
    if (n_paths == 0) return VRT_OK;
    if (integrator == VRT_PI_MC_COLLISION) {
        k_collision_mc_fw<<<grid_blocks(n_paths, num_sms), 256, 0, stream>>>(M, S, n_paths, seed,
                                                                                                out, scale, sc);
    } else {
        cudaError_t e = cudaMemsetAsync(&sc->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        k_collision_dda_fw<<<lane_blocks((const void*)k_collision_dda_fw, n_paths, num_sms), 256, 0, stream>>>(
            M, S, n_paths, seed, out, scale, sc);
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_collision_bw(const DMedium& M, int integrator, const PathSrc& S, uint64_t n_paths, uint64_t seed,
                        const float* dL, float div, DScratch* sc, int num_sms, cudaStream_t stream) {
    if (n_paths == 0) return VRT_OK;
    if (integrator == VRT_PI_MC_COLLISION) {
        k_collision_mc_bw<<<grid_blocks(n_paths, num_sms), 256, 0, stream>>>(M, S, n_paths, seed,
                                                                                                dL, div, sc);
    } else {
        cudaError_t e = cudaMemsetAsync(&sc->next_path, 0, sizeof(unsigned long long), stream);
        if (e != cudaSuccess) return launch_status(e);
        k_collision_dda_bw<<<lane_blocks((const void*)k_collision_dda_bw, n_paths, num_sms), 256, 0, stream>>>(
            M, S, n_paths, seed, dL, div, sc);
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_collision_sample(const DMedium& M, const float* rays, int64_t n, uint64_t seed, float* out3,
                            const float* dL3, DScratch* sc, int num_sms, cudaStream_t stream) {
    if (n == 0) return VRT_OK;
    const int g = grid_blocks((uint64_t)n, num_sms);
    if (out3) k_collision_sample_fw<<<g, 256, 0, stream>>>(M, rays, n, seed, out3, sc);
    else k_collision_sample_bw<<<g, 256, 0, stream>>>(M, rays, n, seed, dL3, sc);
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
