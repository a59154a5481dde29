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
//   k_shadow_run transmittance of each job with the job's own Philox fork,
//                then out[pixel] += weight * T (k_shadow_fw: the DDA form).
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
// path is done.  An uncapped path (the reference's default) walks at most
// kUncappedPass vertices in a round; then its state at the start of its next
// segment (position, direction, throughput, emission sum, stream position)
// is saved and the next round resumes it before taking new paths, so it
// draws exactly what the sequential definition draws.
//
// This file also holds the shadow kernels of the NEE_DS adjoint wavefront
// (vrt_wave_ds.cu): ratio / delta tracking as persistent kernels that advance
// every lane one step per iteration and refill finished lanes from the job
// buffer, and the per-job DDA forms.
#include "vrt_wave.cuh"

namespace vrt {

using namespace wave;


struct WaveFw {
    ShadowJob* jobs;
    unsigned long long* count;
    unsigned long long cap, reserve;
    int cut;          // >= 0: paths stop into the radiance cache at their (cut+1)-th real collision
    float* q;         // the cache queries: 3 planes [rows, 3] (position, direction, throughput)
    long long rows;
    // uncapped paths: after kpass vertices in a pass a path's state at the
    // start of its next segment is saved (5 float4: x, w, W, the emission
    // sum, pid, bounces and the stream position) and resumed in the next
    // round, before new paths; kpass == 0 with a bounce cap or a cut
    int kpass;
    const float4* cin;
    unsigned long long n_cin;
    unsigned long long* cin_head;
    float4* cout;
    unsigned long long* cout_count;
    unsigned long long cap_cont, lanes;
};

// FULL: uncapped passes, the radiance-cache cut and image environments; the
// host launches the FULL = false instance when the medium and call need none
// of them.
template <bool FULL>
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
    int pass_verts = 0;  // vertices of the current path in this pass (uncapped paths)
    bool alive = false, exhausted = false;
    uint32_t n_paths_done = 0, n_verts = 0;
    // the job slot reserved for the direct term of the lane's next path (taken
    // with the collision jobs of an iteration, so a path start needs no scan of
    // its own; ~0: none yet)
    unsigned long long dslot = ~0ull;
    Tally tl;

    while (true) {
        // ---- refill dead lanes while the job buffer has room for the worst case
        int njobs = 0;
        float3 jx = f3(0.0f), jd = f3(0.0f), jw = f3(0.0f), jw2 = f3(0.0f);
        uint32_t jfork = 0;
        unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            const unsigned nw = (unsigned)__popc(want);
            // saved paths are resumed first (nres of the lanes), new paths fill the rest
            unsigned long long base = 0, rb = 0;
            unsigned nres = 0;
            if ((int)lane == leader) {
                const unsigned long long used = *((volatile unsigned long long*)wv.count);
                bool room = used + wv.reserve <= wv.cap;
                if (FULL && room && wv.kpass > 0)
                    room = *((volatile unsigned long long*)wv.cout_count) + wv.lanes <= wv.cap_cont;
                if (!room) {
                    base = ~0ull;
                } else {
                    if (FULL && wv.n_cin && *((volatile unsigned long long*)wv.cin_head) < wv.n_cin) {
                        rb = atomicAdd(wv.cin_head, (unsigned long long)nw);
                        if (rb < wv.n_cin) nres = (unsigned)(wv.n_cin - rb < nw ? wv.n_cin - rb : nw);
                    }
                    base = nres < nw ? atomicAdd(&sc->next_path, (unsigned long long)(nw - nres)) : 0ull;
                }
            }
            base = __shfl_sync(kAll, base, leader);
            rb = __shfl_sync(kAll, rb, leader);
            nres = __shfl_sync(kAll, nres, leader);
            const unsigned rank = __popc(want & ((1u << lane) - 1u));
            if (base == ~0ull) {
                exhausted = true;  // no room this round: finish the lanes in flight
            } else if (!alive && !exhausted && rank < nres) {
                // resume a saved path at the start of its next segment
                const float4* c = wv.cin + 5 * (rb + rank);
                const float4 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3], c4 = c[4];
                x = make_float3(c0.x, c0.y, c0.z);
                w = make_float3(c0.w, c1.x, c1.y);
                W = make_float3(c1.z, c1.w, c2.x);
                Rem = make_float3(c2.y, c2.z, c2.w);
                pid = (uint64_t)__float_as_uint(c3.x) | ((uint64_t)__float_as_uint(c3.y) << 32);
                bounces = (int)__float_as_uint(c3.z);
                rng.init(seed, pid, 0);
                rng.seek(Rng::Pos{__float_as_uint(c3.w), __float_as_uint(c4.x)});
                float tMin;
                boundary(M, x, w, tMin, d);
                ff = Flight();
                steps_path = 0;
                pass_verts = 0;
                alive = true;
            } else if (!alive && !exhausted) {
                const uint64_t p = base + (rank - nres);
                if (p >= n_paths) {
                    exhausted = true;
                } else {
                    // path_integrator_NEE prologue (vr_path_integrator_NEE.h:3-14): the
                    // direct term T(x0, w0) * E becomes a job on fork 0
                    pid = p;
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    start_ray(S, pid, rng, x0, w0, sc);
                    float tMin, tMax;
                    boundary(M, x0, w0, tMin, tMax);
                    x = x0 + w0 * tMin;
                    w = w0;
                    d = tMax - tMin;
                    W = f3(1.0f);
                    Rem = f3(0.0f);
                    bounces = 0;
                    steps_path = 0;
                    pass_verts = 0;
                    ff = Flight();
                    ++n_paths_done;
                    if (wv.cut >= 0) {  // no query unless the path reaches the cut
                        float* q = wv.q + 3 * pid;
                        q[0] = q[1] = q[2] = 0.0f;
                        q[3 * wv.rows] = q[3 * wv.rows + 1] = 0.0f;
                        q[3 * wv.rows + 2] = 1.0f;
                        q[6 * wv.rows] = q[6 * wv.rows + 1] = q[6 * wv.rows + 2] = 0.0f;
                    }
                    const uint32_t f = rng.ntr++;
                    if (dslot != ~0ull) {
                        put_job(wv.jobs, dslot, x, w, env_radiance_t<FULL>(M, w), job_key(pid, f));
                        dslot = ~0ull;
                    } else {
                        njobs = 1;
                        jx = x;
                        jd = w;
                        jw = env_radiance_t<FULL>(M, w);
                        jfork = f;
                    }
                    alive = d > EPS;
                }
            }
        }
        {  // direct-term jobs of the lanes that had no reserved slot (their first path)
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
                if (ff.tau > md * m) {  // crosses the brick face (optical depth > majorant x distance)
                    x = x + w * md;
                    d -= md;
                    ff.cross(m, md);
                    ff.bk.advance(M);
                    if (!(d > EPS)) { ev = 2; break; }
                    if (k + 1 >= kWalkCross) break;  // the flight resumes in the next iteration
                    continue;
                }
                t = ff.tau / m;
                x = x + w * gmin(t, md);
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
            if (FULL && ev == 1 && wv.cut >= 0 && bounces == wv.cut) {  // the rest of the path comes from the cache
                ++n_verts;
                float* q = wv.q + 3 * pid;
                q[0] = x.x; q[1] = x.y; q[2] = x.z;
                q[3 * wv.rows] = w.x; q[3 * wv.rows + 1] = w.y; q[3 * wv.rows + 2] = w.z;
                q[6 * wv.rows] = W.x; q[6 * wv.rows + 1] = W.y; q[6 * wv.rows + 2] = W.z;
                ev = 2;
            } else if (ev == 1) {  // real collision (vr_path_integrator_NEE.h:41-62)
                ++n_verts;
                const float3 sa = albedo(M, x, tl);
                Rem = Rem + W * (f3(1.0f) - sa) * M.emission;
                W = W * sa;
                float3 wnee;
                const float3 pay = environment_sample_t<FULL>(M, rng, wnee);
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
                // an uncapped path past the pass's vertex budget goes on while the job
                // buffer holds every lane's worst case plus one more vertex per lane;
                // else it is saved for the next round
                if (FULL && ev == 0 && wv.kpass > 0 && ++pass_verts >= wv.kpass &&
                    *((volatile unsigned long long*)wv.count) + wv.reserve + wv.lanes * (unsigned long long)njobs >
                        wv.cap) {
                    const unsigned long long o = atomicAdd(wv.cout_count, 1ull);
                    if (o < wv.cap_cont) {
                        float4* c = wv.cout + 5 * o;
                        c[0] = make_float4(x.x, x.y, x.z, w.x);
                        c[1] = make_float4(w.y, w.z, W.x, W.y);
                        c[2] = make_float4(W.z, Rem.x, Rem.y, Rem.z);
                        c[3] = make_float4(__uint_as_float((uint32_t)pid), __uint_as_float((uint32_t)(pid >> 32)),
                                           __uint_as_float((uint32_t)bounces), __uint_as_float(rng.n));
                        c[4] = make_float4(__uint_as_float(rng.ntr), 0.0f, 0.0f, 0.0f);
                    } else {
                        guard(sc, 11);
                    }
                    alive = false;
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
        {  // the collision's light jobs, and a direct-term slot for the lane's next path
            const int nd = (dslot == ~0ull && !exhausted) ? 1 : 0;
            const unsigned long long slot = reserve_slots(wv.count, njobs + nd);
            if (njobs) {
                put_job(wv.jobs, slot, jx, jd, jw, job_key(pid, jfork));
                if (njobs == 2) put_job(wv.jobs, slot + 1, jx, M.sun_dir, jw2, job_key(pid, jfork + 1));
            }
            if (nd) dslot = slot + (unsigned long long)njobs;
        }
    }
    if (dslot != ~0ull) {  // an unused reserved slot: a ray that misses the medium and adds nothing
        const float nan = __int_as_float(0x7fc00000);
        put_job(wv.jobs, dslot, f3(nan), f3(nan), f3(0.0f), 0ull);
    }
    flush_counters(sc, VRT_K_WALK_FW, n_paths_done, n_verts, tl);
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
    flush_counters(sc, VRT_K_SHADOW_FW, 0, 0, tl);
}

// ---------------------------------------------------------------------------
// Persistent shadow kernels for ratio / delta tracking: one event per lane per
// iteration, finished lanes refilled from the job buffer (a warp claims 128
// jobs per atomic and hands them out by ballot rank).
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
    unsigned long long n = *count;
    if (n > cap) n = cap;
    ShadowRay s;
    JobView jv;
    bool alive = false, exhausted = false;
    WarpQueue wq;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            unsigned long long i;
            const bool got = wq.take(head, n, 128, want, i);  // 128 jobs per warp and atomic
            if (!alive && !exhausted) {
                if (!got) {
                    exhausted = wq.drained;
                } else {
                    jv = get_job(jobs, i);
                    if (OUT == OUT_RECORD && jv.tgt == kAdjOnly) {
                        alive = false;  // an adjoint-only job: nothing to estimate here
                    } else {
                        alive = shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork);
                        if (!alive) shadow_finish<OUT>(S, so, jv, 1.0f);
                    }
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
    flush_counters(sc, OUT == OUT_IMAGE ? VRT_K_SHADOW_FW : VRT_K_SHADOW_T, 0, 0, tl);
}

constexpr int kKeep = 8;  // first-pass collisions a transmittance adjoint keeps (k_shadow_adj)

// The transmittance adjoints of the NEE_DS primal's light jobs
// (vr_transmittance_RT.h:51-141 / _DT.h:30-90): the first pass runs as events
// and keeps its tracking collisions; the reference's second pass replays the
// same draws and scatters at exactly those points, so the scatter is done from
// the kept list once the first pass's estimate is known (a ray with more than
// kKeep collisions replays its second pass as events instead).  dL/dT of a
// light job is dL/dR of its pixel (/ div) dotted with the job's weight
// W * L * phase -- the operands the log replay recomputes for the vertex bit
// for bit -- so this kernel needs nothing from the replay.  No adjoint runs
// for rays from or after a singular (zero-density) vertex, where the
// reference's replay stops (vr_path_integrator_NEE_DS.h:153-154), nor for
// paths the state machine runs (first-collision word kSpilled).  MODE
// ADJ_DRT: the jobs of the DRT adjoint (vr_path_integrator_NEE_DRT.h:68-69,
// 165-167): every job has an adjoint, drawn from fork j of the adjoint's own
// stream 1.  ADJ_SPS: the same for the SPS adjoint (_NEE_SPS.h:115-116,
// 228-234), whose rays after the singular vertex (record word bit 1) weigh
// dL/dT by that vertex's sigma (per path in aux[k].w).
template <int TR, int MODE>
__global__ void __launch_bounds__(256, 4) k_shadow_adj(DMedium M, PathSrc S, const ShadowJob* __restrict__ jobs,
                                                     const unsigned long long* __restrict__ count,
                                                     unsigned long long cap, unsigned long long* head, uint64_t seed,
                                                     const float* __restrict__ info, uint64_t p_begin,
                                                     const float* __restrict__ dL, float div, DScratch* sc,
                                                     const float4* __restrict__ aux) {
    unsigned long long n = *count;
    if (n > cap) n = cap;
    ShadowRay s;
    JobView jv;
    float4 keep[kKeep];  // position, majorant
    float keepf[kKeep];  // RT: r; DT: Pc
    int nkeep = 0, phase = 0;  // 0 idle, 1 first pass, 2 second pass (more than kKeep collisions)
    float outT = 0.0f, dLdT = 0.0f;
    bool exhausted = false;
    WarpQueue wq;
    Tally tl;
    while (true) {
        const unsigned want = __ballot_sync(kAll, phase == 0 && !exhausted);
        if (want) {
            unsigned long long i;
            const bool got = wq.take(head, n, 128, want, i);  // 128 jobs per warp and atomic
            if (phase == 0 && !exhausted) {
                if (!got) {
                    exhausted = wq.drained;
                } else {
                    jv = get_job(jobs, i);
                    dLdT = 0.0f;
                    if ((MODE != ADJ_DS || !(jv.tgt & 2u)) &&
                        __float_as_uint(info[8 * (jv.pid - p_begin) + 7]) != kSpilled) {
                        dLdT = dot(ld3(dL + 3 * out_index(S, jv.pid)) / div, jv.wt);
                        if (MODE == ADJ_SPS && jv.tgt != kAdjOnly && (jv.tgt & 2u)) dLdT *= aux[jv.pid - p_begin].w;
                    }
                    nkeep = 0;
                    if (dLdT != 0.0f && shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork, MODE != ADJ_DS ? 1u : 0u))
                        phase = 1;
                }
            }
        }
        if (__all_sync(kAll, phase == 0 && exhausted)) break;
        if (phase != 0) {
            bool hit;
            float hm, hf;
            const bool done = shadow_event<TR, true>(M, s, tl, sc, hit, hm, hf);
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
                        shadow_begin(M, s, jv.x, jv.dir, seed, jv.pid, jv.fork, MODE != ADJ_DS ? 1u : 0u);
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
    flush_counters(sc, VRT_K_SHADOW_ADJ, 0, 0, tl);
}

// Host: rounds of walk + shadow until every path has been taken.
int launch_wave_fw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed, float* out,
                   float scale, cudaStream_t stream, int cut, float* queries) {
    if (n_paths == 0) return 0;
    if (cut >= 0 && !queries) return VRT_E_NULL_POINTER;
    const unsigned long long lights = M.has_sun ? 2ull : 1ull;
    // light jobs come from the vertices before the cap or the cut; an uncapped
    // path walks at most kUncappedPass vertices per pass and resumes later
    unsigned long long verts = M.max_bounces > 0 ? (unsigned long long)M.max_bounces : ~0ull;
    if (cut >= 0 && (unsigned long long)cut < verts) verts = (unsigned long long)cut;
    const int kpass = verts == ~0ull ? kUncappedPass : 0;
    if (kpass) verts = (unsigned long long)kpass;
    const unsigned long long per_path = 1ull + lights * verts;
    const bool full = kpass > 0 || cut >= 0 || M.env_mode != 0 || M.env_sampler != 0;
    const void* walk = full ? (const void*)k_walk_fw<true> : (const void*)k_walk_fw<false>;
    int blocks = persistent_blocks(walk, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)need;
    // the worst case of every path in flight, plus room for a round's expected jobs
    unsigned long long inflight = (unsigned long long)blocks * 256ull;
    if (inflight > n_paths) inflight = n_paths;
    const unsigned long long reserve = inflight * (per_path + 1);  // + the reserved direct-term slot
    const unsigned long long cap = reserve + batch_jobs(n_paths, 1ull + lights, ctx->batch_limit);
    // saved-path buffers (two, swapped per round): every lane in flight may save once more
    const unsigned long long cap_cont = kpass ? 4ull * (unsigned long long)blocks * 256ull : 0ull;
    const size_t o_cont = 256 + cap * sizeof(ShadowJob), cont_bytes = (size_t)cap_cont * 5 * sizeof(float4);
    int st = ensure_wave_buffer(ctx, o_cont + 2 * cont_bytes);
    if (st) return st;
    WaveFw wv;
    // header words: [0] jobs written, [1] shadow-kernel head, [2] resume head, [3] / [4] saved-path counts
    unsigned long long* hdr = reinterpret_cast<unsigned long long*>(ctx->wave);
    wv.count = hdr;
    wv.jobs = reinterpret_cast<ShadowJob*>(static_cast<char*>(ctx->wave) + 256);
    wv.cap = cap;
    wv.reserve = reserve;
    wv.cut = cut;
    wv.q = queries;
    wv.rows = (long long)n_paths;
    wv.kpass = kpass;
    wv.cap_cont = cap_cont;
    wv.lanes = (unsigned long long)blocks * 256ull;
    float4* cont[2] = {reinterpret_cast<float4*>(static_cast<char*>(ctx->wave) + o_cont),
                       reinterpret_cast<float4*>(static_cast<char*>(ctx->wave) + o_cont + cont_bytes)};
    int side = 0;
    wv.cin = cont[1];
    wv.n_cin = 0;
    wv.cin_head = hdr + 2;
    wv.cout = cont[0];
    wv.cout_count = hdr + 3;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    const int sblocks = ctx->num_sms * 8;
    const int rblocks = persistent_blocks(M.tr_mode == 0 ? (const void*)k_shadow_run<0, OUT_IMAGE>
                                                         : (const void*)k_shadow_run<1, OUT_IMAGE>, 256, ctx->num_sms);
    const ShadowOut so = {out, scale, nullptr, nullptr, 0};
    for (int round = 0;; ++round) {
        // count of the jobs written, the head the persistent shadow kernel takes
        // them from, the resume head and this round's saved-path count
        if ((e = cudaMemsetAsync(hdr, 0, 3 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        if ((e = cudaMemsetAsync(wv.cout_count, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        {
            KernelScope ks(VRT_K_WALK_FW, stream);
            if (full) k_walk_fw<true><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, ctx->scratch, wv);
            else k_walk_fw<false><<<blocks, 256, 0, stream>>>(M, src, n_paths, seed, out, scale, ctx->scratch, wv);
        }
        {
            KernelScope ks(VRT_K_SHADOW_FW, stream);
            switch (M.tr_mode) {
                case 0: k_shadow_run<0, OUT_IMAGE><<<rblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, wv.cap, wv.count + 1, seed, so, ctx->scratch); break;
                case 1: k_shadow_run<1, OUT_IMAGE><<<rblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, wv.cap, wv.count + 1, seed, so, ctx->scratch); break;
                case 2: k_shadow_fw<2><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
                case 3: k_shadow_fw<3><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
                case 4: k_shadow_fw<4><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
                default: k_shadow_fw<5><<<sblocks, 256, 0, stream>>>(M, src, wv.jobs, wv.count, seed, out, scale, ctx->scratch); break;
            }
        }
        count_launches(2);
        if ((st = launch_status(cudaGetLastError()))) return st;
        unsigned long long taken = 0, saved = 0;
        if ((e = cudaMemcpyAsync(&taken, &ctx->scratch->next_path, sizeof(taken), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return launch_status(e);
        if (kpass &&
            (e = cudaMemcpyAsync(&saved, wv.cout_count, sizeof(saved), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
            return launch_status(e);
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
        if (saved > cap_cont) return VRT_E_ITER_CAP;  // (the admission test keeps this from happening)
        if (taken >= n_paths && saved == 0) break;
        if (round > (1 << 20)) return VRT_E_ITER_CAP;
        // the paths saved this round are resumed in the next
        wv.cin = cont[side];
        wv.n_cin = saved;
        side ^= 1;
        wv.cout = cont[side];
        wv.cout_count = hdr + 3 + side;
    }
    return 0;
}

// One job per thread for the DDA and grid-tracking forms: T into the record
// and the path's R / Rsp, then the DDA adjoint with dL/dT as in
// k_shadow_adj (GRT / GDT have no backward).
template <int TR>
__global__ void __launch_bounds__(256, 4) k_shadow_T(DMedium M, PathSrc S, WaveBw wv, uint64_t seed,
                                                   const float* __restrict__ dL, float div, DScratch* sc) {
    unsigned long long n = wv.hdr[0];
    if (n > wv.cap_jobs) n = wv.cap_jobs;
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
        float* io = wv.info + 8 * (jv.pid - wv.p_begin);
        if (c3.x != 0.0f || c3.y != 0.0f || c3.z != 0.0f) {
            float* o = io + ((jv.tgt & 2u) ? 3 : 0);
            atomicAdd(o + 0, c3.x);
            atomicAdd(o + 1, c3.y);
            atomicAdd(o + 2, c3.z);
        }
        if ((TR == 2 || TR == 3) && !(jv.tgt & 2u) && __float_as_uint(io[7]) != kSpilled) {
            const float dLdT = dot(ld3(dL + 3 * out_index(S, jv.pid)) / div, jv.wt);
            transmittance_dda_bw<TR == 3>(M, jv.x, jv.dir, dLdT, tl);
        }
    }
    flush_counters(sc, VRT_K_SHADOW_T, 0, 0, tl);
}

int launch_shadow_record(const DMedium& M, const PathSrc& src, const WaveBw& wv, uint64_t seed, const float* dL,
                         float div, DScratch* sc, int num_sms, cudaStream_t stream) {
    const ShadowOut so = {nullptr, 0.0f, wv.recs, wv.info, wv.p_begin};
    KernelScope ks(VRT_K_SHADOW_T, stream);
    switch (M.tr_mode) {
        case 0:
            k_shadow_run<0, OUT_RECORD><<<persistent_blocks((const void*)k_shadow_run<0, OUT_RECORD>, 256, num_sms), 256,
                                          0, stream>>>(M, src, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[3], seed, so, sc);
            break;
        case 1:
            k_shadow_run<1, OUT_RECORD><<<persistent_blocks((const void*)k_shadow_run<1, OUT_RECORD>, 256, num_sms), 256,
                                          0, stream>>>(M, src, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[3], seed, so, sc);
            break;
        case 2: k_shadow_T<2><<<num_sms * 8, 256, 0, stream>>>(M, src, wv, seed, dL, div, sc); break;
        case 3: k_shadow_T<3><<<num_sms * 8, 256, 0, stream>>>(M, src, wv, seed, dL, div, sc); break;
        case 4: k_shadow_T<4><<<num_sms * 8, 256, 0, stream>>>(M, src, wv, seed, dL, div, sc); break;
        default: k_shadow_T<5><<<num_sms * 8, 256, 0, stream>>>(M, src, wv, seed, dL, div, sc); break;
    }
    count_launches(1);
    return launch_status(cudaGetLastError());
}

int launch_shadow_adjoint(const DMedium& M, const PathSrc& src, const WaveBw& wv, uint64_t seed, const float* dL,
                          float div, DScratch* sc, int num_sms, cudaStream_t stream, int mode) {
    if (M.tr_mode > 1) return VRT_OK;  // DDA: in k_shadow_T; GRT / GDT: no backward
    KernelScope ks(VRT_K_SHADOW_ADJ, stream);
#define VRT_ADJ(TR, D)                                                                                             \
    k_shadow_adj<TR, D><<<persistent_blocks((const void*)k_shadow_adj<TR, D>, 256, num_sms), 256, 0, stream>>>( \
        M, src, wv.jobs, &wv.hdr[0], wv.cap_jobs, &wv.hdr[4], seed, wv.info, wv.p_begin, dL, div, sc, wv.resv)
    if (M.tr_mode == 0) {
        if (mode == ADJ_DRT) VRT_ADJ(0, ADJ_DRT);
        else if (mode == ADJ_SPS) VRT_ADJ(0, ADJ_SPS);
        else VRT_ADJ(0, ADJ_DS);
    } else {
        if (mode == ADJ_DRT) VRT_ADJ(1, ADJ_DRT);
        else if (mode == ADJ_SPS) VRT_ADJ(1, ADJ_SPS);
        else VRT_ADJ(1, ADJ_DS);
    }
#undef VRT_ADJ
    count_launches(1);
    return launch_status(cudaGetLastError());
}

}  // namespace vrt
