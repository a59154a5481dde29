// vrt_wave_ds.cu -- the NEE_DS adjoint as a wavefront (sm_100a).
//
// Compiled with -fmad=false: the primal walk (k_ds_primal) and the replay walk
// of the paths the collision log could not hold (k_ds_rewalk) are separate
// kernels that must retrace the same path bit for bit, and the log replay
// (k_ds_replay) must redo the primal's throughput arithmetic exactly, so every
// operation is rounded on its own and no a*b+c can be contracted differently
// in them.  The shadow kernels of the rounds live in vrt_wave.cu.
#include "vrt_wave.cuh"

namespace vrt {

using namespace wave;

// ------------------------------------------------------------------------
// NEE_DS adjoint (include/vr_path_integrator_NEE_DS.h:6-206) as a wavefront.
//
// With the default replay majorant (the primal's) the reference's replay
// retraces the primal's vertices exactly -- same draws, same throughputs, and
// shadow j of the path draws from fork j in both passes.  So the primal logs
// what the replay would recompute: a 32-byte collision record per tracking
// collision and a 48-byte vertex record per scattering vertex; a vertex's
// shadow transmittances are computed once into its record, and the
// transmittance adjoints (which feed nothing back into the path) run over the
// primal's light jobs (same rays, same forks) right after their T:
//
//   A k_ds_primal   the primal walk: per tracking collision a collision record,
//                   per real collision a vertex record (both linked per path)
//                   and a T job per light; per path the emission and escape
//                   terms of R and Rsp
//   B (vrt_wave.cu) T of each job into its record, weight * T into its
//                   path's R (or Rsp after a zero-density collision); then
//                   each job's transmittance adjoint (ratio / delta tracking
//                   or DDA) with dL/dT = dL/dR(pixel) / div . weight -- from
//                   the operands the replay would use for the vertex; none
//                   from or after a singular vertex, where the replay stops
//   C k_ds_replay   the replay from the log: dL/dsigma at every collision,
//                   dL/dalbedo at real ones, the R bookkeeping from the stored T
//     k_ds_rewalk   the same for the paths the log had no room for, by walking
//                   them again with the primal's draws
//
// Rounds bound the buffers as in the forward wavefront.
// ------------------------------------------------------------------------

// FULL: uncapped passes and image environments (the FULL = false instance
// serves the capped walks under a constant environment).
template <bool FULL>
__global__ void __launch_bounds__(256, 3) k_ds_primal(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
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
    // a path's records are linked forward without patching: each record is
    // written with the slot reserved for the path's next one (rec_next,
    // ev_next), so every path leaves one reserved slot of each kind unused
    uint32_t steps_path = 0, first = kNone, rec_next = kNone, first_ev = kNone, ev_next = kNone, n_ev = 0;
    uint32_t n_paths_done = 0;
    bool logged = false, spilled = false;
    Tally tl;

    while (true) {
        unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) {
                const unsigned long long uj = *((volatile unsigned long long*)&wv.hdr[0]);
                const unsigned long long ur = *((volatile unsigned long long*)&wv.hdr[1]);
                const unsigned long long ue = *((volatile unsigned long long*)&wv.hdr[5]);
                const unsigned long long up = *((volatile unsigned long long*)&sc->next_path) - wv.p_begin;
                const bool room = uj + wv.res_jobs <= wv.cap_jobs && ur + wv.res_recs <= wv.cap_recs &&
                                  ue + wv.res_evs <= wv.cap_evs && up + wv.lanes <= wv.cap_paths;
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
                    start_ray(S, pid, rng, x0, w0, sc);
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
                    rec_next = kNone;
                    first_ev = kNone;
                    ev_next = kNone;
                    n_ev = 0;
                    logged = true;
                    spilled = false;
                    ff = Flight();
                    alive = true;
                    ++n_paths_done;
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        int nrec = 0, nj = 0, nev = 0;
        bool finish = false, rsp = false;
        float3 wnee = f3(0.0f), sa = f3(0.0f), Le = f3(0.0f);
        float ev_s = 0.0f, ev_m = 0.0f, ph_env = 0.0f, ph_sun = 0.0f;
        uint32_t jfork = 0, ev_real = 0;
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
                    if (ff.tau > md * m) {  // crosses the brick face (optical depth > majorant x distance)
                        x = x + w * md;
                        d -= md;
                        ff.cross(m, md);
                        ff.bk.advance(M);
                        if (!(d > EPS)) { ev = 2; break; }
                        if (k + 1 >= kDsCross) break;  // the flight resumes in the next iteration
                        continue;
                    }
                    t = ff.tau / m;
                    x = x + w * gmin(t, md);
                    ff.used();
                    if (t > d) ev = 2;
                    else need = true;
                    ff.bk.move(t);
                    break;
                }
                if (need) {
                    const float s = sigma(M, x, tl);
                    const float Pc = (s + eps) / m;
                    nev = logged ? (ev_next == kNone ? 2 : 1) : 0;  // this collision's slot and the next one's
                    ev_s = s;
                    ev_m = m;
                    if (rng.uniform() >= Pc) {  // null collision (_NEE_DS.h:41-45)
                        W = W * ((1.0f - s / m) / (1.0f - Pc));
                        d -= t;
                    } else {  // real collision (_NEE_DS.h:48-99)
                        ev_real = 1u;
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
                            sa = albedo(M, x, tl);
                            const float3 acc = W * (f3(1.0f) - sa) * M.emission;
                            W = W * sa;
                            Le = environment_sample_t<FULL>(M, rng, wnee);
                            ph_env = phase(M, w, wnee);
                            if (M.has_sun) ph_sun = phase(M, w, M.sun_dir);
                            jfork = rng.ntr;
                            rng.ntr += (uint32_t)lights;
                            const bool capped = M.max_bounces > 0 && bounces + 1 >= M.max_bounces;
                            // an uncapped path past the pass's vertex budget goes on while the
                            // buffers hold every lane's worst case plus one more vertex per lane
                            // (at most one such approval per lane is ever outstanding); else it
                            // goes to the state machine
                            bool at_budget = FULL && wv.kpass > 0 && bounces + 1 >= wv.kpass;
                            if (at_budget) {
                                const unsigned long long uj = *((volatile unsigned long long*)&wv.hdr[0]);
                                const unsigned long long ur = *((volatile unsigned long long*)&wv.hdr[1]);
                                at_budget = !(uj + wv.res_jobs + wv.lanes * (unsigned long long)lights <= wv.cap_jobs &&
                                              ur + wv.res_recs + wv.lanes * 2ull <= wv.cap_recs);
                            }
                            float3 wo = w;
                            if (!capped && !at_budget) wo = phase_sample(M, rng, w);
                            rsp = null_W < EPS;
                            if (rsp) Rspacc = Rspacc + acc;
                            else Racc = Racc + acc;
                            nrec = rec_next == kNone ? 2 : 1;
                            nj = lights;
                            ++bounces;
                            if (capped || all_less(W, EPS)) {
                                ev = 2;  // W stays: the light jobs below weigh with it
                            } else if (at_budget) {
                                ev = 2;
                                spilled = true;
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
        // ---- one reservation for the T jobs, the vertex record, the collision
        // record and (at the end of a path with logged collisions) its replay-list entry
        const int nl = (finish && logged && !spilled && (first_ev != kNone || nev)) ? 1 : 0;
        const Slots4 sl = reserve_slots4(&wv.hdr[0], &wv.hdr[1], &wv.hdr[5], &wv.hdr[8],
                                         (uint32_t)nj | ((uint32_t)nrec << 8) | ((uint32_t)nev << 16) |
                                             ((uint32_t)nl << 24));
        const unsigned long long r = rec_next == kNone ? sl.s1 : rec_next;
        if (nrec) {  // the vertex record, with the slot of the path's next one
            const uint32_t rn = rec_next == kNone ? (uint32_t)(sl.s1 + 1) : (uint32_t)sl.s1;
            uint4* rp = reinterpret_cast<uint4*>(wv.recs + r);
            __stcs(rp, make_uint4(__float_as_uint(1.0f), __float_as_uint(1.0f), rn, (uint32_t)sl.s0));
            __stcs(reinterpret_cast<float4*>(rp + 1), make_float4(sa.x, sa.y, sa.z, ph_env));
            __stcs(reinterpret_cast<float4*>(rp + 2), make_float4(Le.x, Le.y, Le.z, ph_sun));
            tl.logb += (uint32_t)sizeof(VertexRec);
            if (first == kNone) first = (uint32_t)r;
            rec_next = rn;
        }
        if (nev) {  // the collision record (null and real), with the slot of the path's next one
            const unsigned long long je = ev_next == kNone ? sl.s2 : ev_next;
            const unsigned long long jn = ev_next == kNone ? sl.s2 + 1 : sl.s2;
            if (je >= wv.cap_evs || jn >= wv.cap_evs) {
                logged = false;  // the log is full: this path is replayed by walking it again
            } else {
                CollisionRec* ep = wv.evs + je;
                __stcs(&ep->xs, make_float4(x.x, x.y, x.z, ev_s));
                __stcs(&ep->link, make_uint4(__float_as_uint(ev_m), (uint32_t)jn, nrec ? (uint32_t)r : kNone, ev_real));
                tl.logb += (uint32_t)sizeof(CollisionRec);
                if (first_ev == kNone) first_ev = (uint32_t)je;
                ev_next = (uint32_t)jn;
                ++n_ev;
            }
        }
        if (nj) {
            const unsigned long long j = sl.s0;
            const uint32_t tgt = ((uint32_t)r << 2) | (rsp ? 2u : 0u);
            // the light rays of the vertex, weighted W * L * phase (W after the albedo)
            put_job(wv.jobs, j, x, wnee, W * Le * ph_env, job_key(pid, jfork), tgt);
            if (nj == 2) put_job(wv.jobs, j + 1, x, M.sun_dir, W * M.sun_L * ph_sun, job_key(pid, jfork + 1), tgt | 1u);
        }
        if (finish) {  // end of the primal (_NEE_DS.h:106-110): escape term, then the path's totals
            if (!scattered) Racc = Racc + env_radiance_t<FULL>(M, w) * W;
            const uint64_t k = pid - wv.p_begin;
            float* io = wv.info + 8 * k;
            __stcs(reinterpret_cast<float4*>(io), make_float4(Racc.x, Racc.y, Racc.z, Rspacc.x));
            __stcs(reinterpret_cast<float4*>(io) + 1,
                   make_float4(Rspacc.y, Rspacc.z, __uint_as_float(first),
                               __uint_as_float(spilled ? kSpilled : (logged ? first_ev : kUnlogged))));
            // an entry whose last collision found the log full is skipped by the replay
            if (nl) __stcs(wv.list + sl.s3, make_uint4((uint32_t)k, logged ? first_ev : kUnlogged, n_ev, 0u));
            if (spilled) {  // its records are ignored; the state machine runs the whole path
                const unsigned long long o = atomicAdd(wv.spill_count, 1ull);
                if (o < wv.cap_spill) wv.spill[o] = (unsigned long long)pid;
                else guard(sc, 10);
            } else if (!logged) {
                const unsigned long long o = atomicAdd(&wv.hdr[6], 1ull);
                if (o < wv.cap_paths) wv.over[o] = (uint32_t)k;
                else guard(sc, 8);
            }
            alive = false;
        }
    }
    flush_counters(sc, VRT_K_DS_PRIMAL, n_paths_done, 0, tl);  // the forward counts the vertices
}

__global__ void __launch_bounds__(256, 3) k_ds_rewalk(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                    const float* __restrict__ dL, float div, DScratch* sc, WaveBw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    const int lights = M.has_sun ? 2 : 1;
    unsigned long long n_over = *((volatile unsigned long long*)&wv.hdr[6]);
    if (n_over > wv.cap_paths) n_over = wv.cap_paths;
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
                const unsigned long long q = base + __popc(want & ((1u << lane) - 1u));
                if (q >= n_over) {
                    exhausted = true;
                } else {
                    const unsigned long long k = wv.over[q];
                    pid = wv.p_begin + k;
                    rng.init(seed, pid, 0);
                    float3 x0, w0;
                    start_ray(S, pid, rng, x0, w0, sc);
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
                    if (ff.tau > md * m) {  // the primal's test (k_ds_primal)
                        x = x + w * md;
                        d -= md;
                        ff.cross(m, md);
                        ff.bk.advance(M);
                        if (!(d > EPS)) { ev = 2; break; }
                        if (k + 1 >= kDsCross) break;  // the flight resumes in the next iteration
                        continue;
                    }
                    t = ff.tau / m;
                    x = x + w * gmin(t, md);
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
                            rng.ntr += (uint32_t)lights;  // the forks of the vertex's light rays
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
                                // (the light rays' transmittance adjoints run with the T jobs)
                                R = R - W * Te * Le * ph_nee;
                                if (M.has_sun) R = R - W * Ts * M.sun_L * ph_sun;
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
    }
    flush_counters(sc, VRT_K_DS_REWALK, 0, 0, tl);
}

// Replay of the logged collisions (_NEE_DS.h:112-206 without the walk): the
// primal logged every tracking collision (position, sigma, majorant) and every
// scattering vertex (albedo, light directions, radiance, phases, fork), so the
// replay redoes the estimator's bookkeeping -- W, R and the scatter weights --
// from the log with the same arithmetic, and no majorant walk, sigma or albedo
// lookup, or random draw.  Lanes take paths from the primal's list of paths
// with logged collisions; each iteration replays one collision per lane while
// the loads of the path's next collision and of the vertex record are in
// flight.
__global__ void __launch_bounds__(256, 3) k_ds_replay(DMedium M, PathSrc S, const float* __restrict__ dL, float div,
                                                    DScratch* sc, WaveBw wv) {
    const float EPS = 0.00000001f;
    const float eps = M.ds_eps;
    unsigned long long n_list = *((volatile unsigned long long*)&wv.hdr[8]);
    if (n_list > wv.cap_paths) n_list = wv.cap_paths;
    float3 W = f3(0.0f), R = f3(0.0f), Rsp = f3(0.0f), dLdR = f3(0.0f);
    bool alive = false, exhausted = false;
    int bounces = 0;
    uint64_t pid = 0;
    uint32_t left = 0;  // collisions of the path still to replay
    float4 xs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // the collision to replay
    uint4 ln = make_uint4(0u, kNone, kNone, 0u);
    WarpQueue wq;
    Tally tl;

    while (true) {
        const unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            unsigned long long q;
            const bool got = wq.take(&wv.hdr[7], n_list, 32, want, q);
            if (!alive && !exhausted) {
                if (!got) {
                    exhausted = wq.drained;
                } else {
                    const uint4 e = __ldcs(wv.list + q);
                    if (e.y != kUnlogged && e.z > 0u) {  // (a path whose last collision found the log full: k_ds_rewalk)
                        const CollisionRec* ep = wv.evs + e.y;
                        xs = __ldcs(&ep->xs);
                        ln = __ldcs(&ep->link);
                        const float4* io = reinterpret_cast<const float4*>(wv.info + 8 * (uint64_t)e.x);
                        const float4 a = io[0], b = io[1];
                        pid = wv.p_begin + e.x;
                        dLdR = ld3(dL + 3 * out_index(S, pid)) / div;
                        R = make_float3(a.x, a.y, a.z);
                        Rsp = make_float3(a.w, b.x, b.y);
                        W = f3(1.0f);
                        bounces = 0;
                        left = e.z;
                        alive = true;
                    }
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        if (alive) {
            bool end = false;
            // the next collision of the path and this one's vertex record, loaded ahead
            const uint32_t nx = ln.y;
            const bool real = (ln.w & 1u) != 0u;
            float4 nxs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            uint4 nln = make_uint4(0u, kNone, kNone, 0u);
            if (left > 1u) {
                const CollisionRec* np = wv.evs + nx;
                nxs = __ldcs(&np->xs);
                nln = __ldcs(&np->link);
            }
            uint4 r0 = make_uint4(0u, 0u, 0u, 0u);
            float4 r1 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), r2 = r1;
            if (real && ln.z != kNone) {
                const uint4* rp = reinterpret_cast<const uint4*>(wv.recs + ln.z);
                r0 = __ldcs(rp);
                r1 = __ldcs(reinterpret_cast<const float4*>(rp + 1));
                r2 = __ldcs(reinterpret_cast<const float4*>(rp + 2));
            }
            tl.logb += (uint32_t)sizeof(CollisionRec);
            ++tl.steps;
            const float3 x = make_float3(xs.x, xs.y, xs.z);
            const float s = xs.w, m = __uint_as_float(ln.x);
            const float Pc = (s + eps) / m;
            float gsc;
            if (!real) {  // _NEE_DS.h:130-140
                gsc = dot(dLdR, -R / m / (1.0f - s / m));
                W = W * ((1.0f - s / m) / (1.0f - Pc));
            } else {      // _NEE_DS.h:142-150
                gsc = dot(dLdR, s < EPS ? Rsp / eps : R / s);
            }
            if (gsc != 0.0f) sigma_bw(M, x, gsc, tl);
            if (real) {   // the scattering vertex (_NEE_DS.h:151-203)
                W = W * (s / m / Pc);
                if (s < EPS || ln.z == kNone) {
                    if (s >= EPS) guard(sc, 9);  // a scattering collision without its vertex record
                    end = true;
                } else {
                    tl.logb += (uint32_t)sizeof(VertexRec);
                    const float Te = __uint_as_float(r0.x), Ts = __uint_as_float(r0.y);
                    const float3 sa = make_float3(r1.x, r1.y, r1.z);
                    const float ph_nee = r1.w, ph_sun = r2.w;
                    const float3 Le = make_float3(r2.x, r2.y, r2.z);
                    float3 dL_dsa = dLdR * W * -1.0f * M.emission;
                    R = R - W * (f3(1.0f) - sa) * M.emission;
                    dL_dsa = dL_dsa + dLdR * R / make_float3(gmax(EPS, sa.x), gmax(EPS, sa.y), gmax(EPS, sa.z));
                    albedo_bw(M, x, dL_dsa, tl);
                    W = W * sa;
                    // the vertex's light rays (their transmittance adjoints ran with the T jobs)
                    R = R - W * Te * Le * ph_nee;
                    if (M.has_sun) R = R - W * Ts * M.sun_L * ph_sun;
                    ++bounces;
                    if ((M.max_bounces > 0 && bounces >= M.max_bounces) || all_less(W, EPS)) end = true;
                }
            }
            xs = nxs;
            ln = nln;
            if (--left == 0u) end = true;
            if (end) alive = false;
        }
    }
    flush_counters(sc, VRT_K_DS_REPLAY, 0, 0, tl);
}

int launch_wave_ds_bw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                      const float* dL, float div, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.ds_compat) return VRT_E_UNSUPPORTED;
    // uncapped paths walk at most kUncappedPass vertices here; the few that go on
    // are run whole by the state machine afterwards
    const int kpass = M.max_bounces > 0 ? 0 : kUncappedPass;
    const unsigned long long lights = M.has_sun ? 2ull : 1ull;
    const unsigned long long B = (unsigned long long)(M.max_bounces > 0 ? M.max_bounces : kpass);
    const bool full = kpass > 0 || M.env_mode != 0 || M.env_sampler != 0;
    int blocksA = persistent_blocks(full ? (const void*)k_ds_primal<true> : (const void*)k_ds_primal<false>, 256,
                                    ctx->num_sms);
    int blocksC = persistent_blocks((const void*)k_ds_replay, 256, ctx->num_sms);
    int blocksW = persistent_blocks((const void*)k_ds_rewalk, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocksA > need) blocksA = (int)need;
    if ((uint64_t)blocksC > need) blocksC = (int)need;
    if ((uint64_t)blocksW > need) blocksW = (int)need;
    WaveBw wv{};
    wv.lanes = (unsigned long long)blocksA * 256ull;
    const unsigned long long inflight = wv.lanes < n_paths ? wv.lanes : n_paths;
    wv.res_jobs = inflight * lights * B;
    wv.res_recs = inflight * (B + 1);  // B records and the reserved slot after the last one
    // room for three vertex records per path (the NEE_DS primal's majorant and
    // epsilon collisions make more vertices than the forward's: 2.3 per path
    // on the benchmark medium)
    wv.cap_jobs = wv.res_jobs + batch_jobs(n_paths, 3ull * lights, ctx->batch_limit);
    wv.cap_recs = wv.res_recs + batch_jobs(n_paths, 3, ctx->batch_limit);
    if (wv.cap_recs > (1ull << 30)) return VRT_E_UNSUPPORTED;  // record indices are 30-bit in a job
    wv.cap_paths = (n_paths < (1ull << 24) ? n_paths : (1ull << 24)) + wv.lanes;
    // the collision log: room for about four collisions per vertex record of a
    // round, and admission of new paths stops while less than 16 collisions per
    // lane in flight are left; a path that still finds it full is re-walked
    wv.cap_evs = ctx->log_limit ? ctx->log_limit : 4ull * batch_jobs(n_paths, 1, ctx->batch_limit) + inflight * 16ull;
    if (wv.cap_evs > 0xfff00000ull) wv.cap_evs = 0xfff00000ull;  // 32-bit links, kNone / kUnlogged reserved
    wv.res_evs = inflight * 16ull < wv.cap_evs / 2 ? inflight * 16ull : wv.cap_evs / 2;
    const size_t o_jobs = 256, o_recs = o_jobs + wv.cap_jobs * sizeof(ShadowJob);
    const size_t o_info = o_recs + wv.cap_recs * sizeof(VertexRec), o_over = o_info + wv.cap_paths * 32;
    const size_t o_list = o_over + ((wv.cap_paths * 4 + 255) & ~(size_t)255);
    const size_t o_evs = o_list + ((wv.cap_paths * 16 + 255) & ~(size_t)255);
    wv.kpass = kpass;
    wv.cap_spill = kpass > 0 ? (unsigned long long)n_paths : 0ull;
    const size_t o_spill = o_evs + wv.cap_evs * 32, bytes = o_spill + wv.cap_spill * 8;
    int st = ensure_wave_buffer(ctx, bytes);
    if (st) return st;
    char* base = static_cast<char*>(ctx->wave);
    wv.hdr = reinterpret_cast<unsigned long long*>(base);
    wv.jobs = reinterpret_cast<ShadowJob*>(base + o_jobs);
    wv.recs = reinterpret_cast<VertexRec*>(base + o_recs);
    wv.info = reinterpret_cast<float*>(base + o_info);
    wv.over = reinterpret_cast<uint32_t*>(base + o_over);
    wv.list = reinterpret_cast<uint4*>(base + o_list);
    wv.evs = reinterpret_cast<CollisionRec*>(base + o_evs);
    wv.spill = reinterpret_cast<unsigned long long*>(base + o_spill);
    wv.spill_count = &wv.hdr[10];  // kept across rounds
    wv.resv = nullptr;
    wv.p_begin = 0;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    if ((e = cudaMemsetAsync(wv.spill_count, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
        return launch_status(e);
    for (int round = 0;; ++round) {
        // [0] jobs, [1] records, [2] re-walk queue, [3] / [4] heads of the shadow kernels,
        // [5] collisions, [6] paths left out of the log, [7] replay-list head, [8] replay list
        if ((e = cudaMemsetAsync(wv.hdr, 0, 9 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        {
            KernelScope ks(VRT_K_DS_PRIMAL, stream);
            if (full) k_ds_primal<true><<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
            else k_ds_primal<false><<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
        }
        // the primal's light jobs: T into the records and paths, then their transmittance adjoints
        if ((st = launch_shadow_record(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream))) return st;
        if ((st = launch_shadow_adjoint(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream))) return st;
        {
            KernelScope ks(VRT_K_DS_REPLAY, stream);
            k_ds_replay<<<blocksC, 256, 0, stream>>>(M, src, dL, div, ctx->scratch, wv);
        }
        {
            // exits at once when every path of the round fit the log
            KernelScope ks(VRT_K_DS_REWALK, stream);
            k_ds_rewalk<<<blocksW, 256, 0, stream>>>(M, src, n_paths, seed, dL, div, ctx->scratch, wv);
        }
        count_launches(3);
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
    if (kpass > 0) {  // the uncapped paths longer than the pass budget, whole, on the state machine
        unsigned long long spilled = 0;
        if ((e = cudaMemcpyAsync(&spilled, wv.spill_count, sizeof(spilled), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return launch_status(e);
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
        if (spilled > wv.cap_spill) spilled = wv.cap_spill;
        if (spilled)
            return launch_nee_ds_bw(M, src, spilled, seed, dL, div, ctx->scratch, ctx->num_sms, stream, wv.spill);
    }
    return 0;
}

}  // namespace vrt
