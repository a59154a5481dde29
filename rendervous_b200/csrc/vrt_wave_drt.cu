// vrt_wave_drt.cu -- the DRT adjoint as a wavefront (sm_100a).
//
// The reference's differential-ratio-tracking adjoint
// (include/vr_path_integrator_NEE_DRT.h:62-270; its DRTDS form,
// _NEE_DRTDS.h:40-253, differs only in the replay's real collisions and the
// branch's position sampler) walks each path three times:
// the primal (majorant x1.05 + 0.1, R from the light rays of every real
// collision, a reservoir vertex kept in proportion to the throughput), the
// replay with the same draws (a sigma scatter at every tracking collision, the
// light rays' transmittance adjoints from the adjoint's own stream 1), and a
// branch from the reservoir vertex.  Nothing the replay computes changes the
// path, so, as for NEE_DS (vrt_wave_ds.cu), the primal logs what the replay
// would recompute:
//
//   k_drt_primal   per tracking collision a 32-byte collision record, per
//                  real collision a vertex record and one job per light, per
//                  path the reservoir vertex and the stream position at its
//                  end; the primary ray's environment adjoint is a job of its
//                  own (kAdjOnly: an adjoint and no T)
//   (vrt_wave.cu)  T of every job into its record and the path's R, then the
//                  jobs' transmittance adjoints from fork j of stream 1 with
//                  dL/dT = dL/dR(pixel) / div . weight -- the fork numbers of
//                  the two streams agree (fork 0 is the primary ray's in both)
//   k_drt_replay   the sigma scatters of the log, R taken down vertex by vertex
//   k_drt_branch_pre / _post (vrt_path.cu) the reservoir branch from the
//                  stream position the primal ended at (the replay draws
//                  exactly the primal's): its position and light rays one
//                  thread per path, its nested scattered-only NEE path on the
//                  state machine (k_nee_fw<FW_BRANCH>), then the scatter
//
// DRTQ (_NEE_DRTQ.h:58-260) is the same primal without the reservoir and the
// same replay; instead of one branch it takes a scatter term on every segment
// (the primary ray and the segment after each scattering vertex that does not
// end the path), each from a stream of its own (Rng::segment_stream), so the
// primal writes the segments (segment 0 in resv, the others in segs) and
// k_drtq_segment_pre + k_nee_fw<FW_BRANCH> + k_drt_branch_post<2>
// (vrt_path.cu) run one term per thread and item.
//
// Compiled with -fmad=false, like the sequential form (vrt_path.cu), so a
// walk here rounds as the sequential definition does.  Paths the collision log
// cannot hold, and uncapped paths still going after kUncappedPass vertices,
// run whole on the sequential form afterwards, over a list of their ids (their
// jobs here are skipped: first-collision word kSpilled).
#include "vrt_wave.cuh"

namespace vrt {

using namespace wave;

template <bool Q>
__global__ void __launch_bounds__(256, 3) k_drt_primal(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                     DScratch* sc, WaveBw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00000001f;
    const int lights = M.has_sun ? 2 : 1;
    Flight ff;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f);
    float d = 0.0f, total_weight = 0.0f;
    bool alive = false, exhausted = false, logged = false;
    int bounces = 0;
    uint64_t pid = 0;
    // records are linked forward through pre-reserved slots, as in k_ds_primal
    uint32_t steps_path = 0, first = kNone, rec_next = kNone, first_ev = kNone, ev_next = kNone, n_ev = 0;
    uint32_t n_paths_done = 0;
    Tally tl;

    while (true) {
        const unsigned want = __ballot_sync(kAll, !alive && !exhausted);
        if (want) {
            unsigned long long jb;
            const unsigned long long base = admit_paths(wv, sc, n_paths, want, jb);
            if (base == ~0ull) {
                exhausted = true;
            } else if (!alive && !exhausted) {
                const unsigned rank = __popc(want & ((1u << lane) - 1u));
                const uint64_t p = base + rank;
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
                    const uint64_t k = pid - wv.p_begin;
                    float4* rv = wv.resv + 4 * k;
                    ++n_paths_done;
                    if (!(d > 0.0f)) {  // _NEE_DRT.h:67: nothing to do, and no branch (total weight 0)
                        put_job(wv.jobs, jb + rank, x, w, f3(0.0f), job_key(pid, 0), kAdjOnly);
                        float* io = wv.info + 8 * k;
                        __stcs(reinterpret_cast<float4*>(io), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
                        __stcs(reinterpret_cast<float4*>(io) + 1,
                               make_float4(0.0f, 0.0f, __uint_as_float(kNone), __uint_as_float(kNone)));
                        if (Q) __stcs(rv, make_float4(x.x, x.y, x.z, 0.0f));  // no scatter term either
                        else __stcs(rv + 1, make_float4(w.x, w.y, w.z, 0.0f));
                    } else {
                        // _NEE_DRT.h:68-69: the primal's T of the primary ray takes fork 0 of the
                        // path's stream (its value is unused); its adjoint, fork 0 of stream 1
                        rng.ntr += 1u;
                        put_job(wv.jobs, jb + rank, x, w, env_radiance(M, w), job_key(pid, 0), kAdjOnly);
                        W = f3(1.0f);
                        total_weight = 3.0f;
                        if (Q) {  // DRTQ: segment 0, the primary ray's, for its scatter term
                            __stcs(rv, make_float4(x.x, x.y, x.z, d));
                            __stcs(rv + 1, make_float4(w.x, w.y, w.z, __uint_as_float(0u)));
                            __stcs(rv + 2, make_float4(1.0f, 1.0f, 1.0f, __uint_as_float((uint32_t)k)));
                        } else {  // the reservoir starts at the primary ray
                            __stcs(rv, make_float4(x.x, x.y, x.z, 3.0f));
                            __stcs(rv + 1, make_float4(w.x, w.y, w.z, 3.0f));
                            __stcs(rv + 2, make_float4(1.0f, 1.0f, 1.0f, 0.0f));
                        }
                        bounces = 0;
                        steps_path = 0;
                        first = kNone;
                        rec_next = kNone;
                        first_ev = kNone;
                        ev_next = kNone;
                        n_ev = 0;
                        logged = true;
                        ff = Flight();
                        alive = true;
                    }
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        int nrec = 0, nj = 0, nev = 0;
        uint32_t nseg = 0;  // DRTQ: the segment after this vertex takes a scatter term
        bool finish = false, spill = false;
        float3 wnee = f3(0.0f), sa = f3(0.0f), Le = f3(0.0f);
        float ev_s = 0.0f, ev_m = 0.0f, ph_env = 0.0f, ph_sun = 0.0f;
        uint32_t jfork = 0, ev_real = 0;
        if (alive) {
            int ev = 0;  // 0 none, 1 collision, 2 end
            if (!(d > EPS)) {
                ev = 2;  // the loop test (_NEE_DRT.h:79)
            } else {
                bool need = false;
                float m = 0.0f, t = 0.0f;
                for (int k = 0;; ++k) {
                    if (k >= kStepCap) {
                        guard(sc, 12);
                        ev = 2;
                        break;
                    }
                    // _NEE_DRT.h:81-86: a brick face crossed when t > md (the sequential form's test)
                    float md;
                    m = ff.bk.query(M, x, w, md) * 1.05f + 0.1f;
                    if (ff.tau < 0.0f) ++tl.steps;
                    t = ff.sample(rng) / m;
                    x = x + w * gmin(t, md);
                    if (t > md) {
                        d -= md;
                        ff.cross(m, md);
                        ff.bk.advance(M);
                        if (!(d > EPS)) { ev = 2; break; }
                        if (k + 1 >= kDsCross) break;  // the flight resumes in the next iteration
                        continue;
                    }
                    ff.used();
                    if (t > d) {
                        ev = 2;
                    } else {
                        need = true;
                        ff.bk.move(t);
                    }
                    break;
                }
                if (need) {
                    const float s = sigma(M, x, tl);
                    nev = logged ? (ev_next == kNone ? 2 : 1) : 0;  // this collision's slot and the next one's
                    ev_s = s;
                    ev_m = m;
                    if (rng.uniform() >= s / m) {  // null collision (_NEE_DRT.h:90)
                        d -= t;
                    } else {  // real collision (_NEE_DRT.h:91-112)
                        ev_real = 1u;
                        sa = albedo(M, x, tl);
                        W = W * sa;
                        Le = environment_sample(M, rng, wnee);
                        ph_env = phase(M, w, wnee);
                        if (M.has_sun) ph_sun = phase(M, w, M.sun_dir);
                        jfork = rng.ntr;  // the forks of the vertex's light rays
                        rng.ntr += (uint32_t)lights;
                        ++bounces;
                        const bool capped = M.max_bounces > 0 && bounces >= M.max_bounces;
                        w = phase_sample(M, rng, w);
                        float tMin;
                        boundary(M, x, w, tMin, d);
                        ff.bk.reset();
                        if (!Q) {  // the reservoir: this vertex replaces the kept one with probability P / total
                            const float current_P = W.x + W.y + W.z;
                            total_weight += current_P;
                            if (rng.uniform() < current_P / total_weight) {
                                float4* rv = wv.resv + 4 * (pid - wv.p_begin);
                                __stcs(rv, make_float4(x.x, x.y, x.z, current_P));
                                __stcs(rv + 1, make_float4(w.x, w.y, w.z, 0.0f));  // total written at the end
                                __stcs(rv + 2, make_float4(W.x, W.y, W.z, 0.0f));
                            }
                        }
                        nrec = rec_next == kNone ? 2 : 1;
                        nj = lights;
                        if (all_less(W, EPS) || capped) {
                            ev = 2;
                        } else if (wv.kpass > 0 && bounces >= wv.kpass) {
                            ev = 2;  // an uncapped path past the pass budget: whole, on the sequential form
                            spill = true;
                        } else if (Q) {
                            nseg = 1u;  // _NEE_DRTQ.h:249-259: the next segment's scatter term
                        }
                    }
                }
            }
            if (++steps_path > (uint32_t)kPathCap) {
                guard(sc, 13);
                ev = 2;
            }
            finish = ev == 2;
        }
        // ---- one reservation for the light jobs, the vertex record, the collision
        // record and (at the end of a path with logged collisions) its replay-list entry
        const int nl = (finish && logged && (first_ev != kNone || nev)) ? 1 : 0;
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
                logged = false;  // the log is full: the path runs whole on the sequential form
                finish = true;
                spill = true;
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
        if (Q) {  // DRTQ: the segment after the vertex (start, direction, throughput, number)
            const Slots4 sq = reserve_slots4(&wv.hdr[14], &wv.hdr[14], &wv.hdr[14], &wv.hdr[14], nseg);
            if (nseg) {
                if (sq.s0 >= wv.cap_segs) {
                    guard(sc, 16);
                } else {
                    float4* g = wv.segs + 3 * sq.s0;
                    __stcs(g, make_float4(x.x, x.y, x.z, d));
                    __stcs(g + 1, make_float4(w.x, w.y, w.z, __uint_as_float((uint32_t)bounces)));
                    __stcs(g + 2, make_float4(W.x, W.y, W.z, __uint_as_float((uint32_t)(pid - wv.p_begin))));
                }
            }
        }
        if (nj) {  // the light rays of the vertex, weighted W * L * phase (W after the albedo)
            const unsigned long long j = sl.s0;
            const uint32_t tgt = (uint32_t)r << 2;
            put_job(wv.jobs, j, x, wnee, W * Le * ph_env, job_key(pid, jfork), tgt);
            if (nj == 2) put_job(wv.jobs, j + 1, x, M.sun_dir, W * M.sun_L * ph_sun, job_key(pid, jfork + 1), tgt | 1u);
        }
        if (finish) {  // the path's words: R (filled by the light rays), first record and collision
            const uint64_t k = pid - wv.p_begin;
            float* io = wv.info + 8 * k;
            __stcs(reinterpret_cast<float4*>(io), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            __stcs(reinterpret_cast<float4*>(io) + 1,
                   make_float4(0.0f, 0.0f, __uint_as_float(first), __uint_as_float(spill ? kSpilled : first_ev)));
            // an entry whose last collision found the log full is skipped by the replay
            if (nl) __stcs(wv.list + sl.s3, make_uint4((uint32_t)k, logged ? first_ev : kUnlogged, n_ev, 0u));
            if (!Q) {
                float4* rv = wv.resv + 4 * k;
                reinterpret_cast<float*>(rv + 1)[3] = total_weight;
                __stcs(rv + 3, make_float4(__uint_as_float(rng.n), __uint_as_float(rng.ntr), 0.0f, 0.0f));
            }
            if (spill) {
                const unsigned long long o = atomicAdd(wv.spill_count, 1ull);
                if (o < wv.cap_spill) wv.spill[o] = (unsigned long long)pid;
                else guard(sc, 14);
            }
            alive = false;
        }
    }
    flush_counters(sc, VRT_K_DRT_PRIMAL, n_paths_done, 0, tl);
}

// The DRT replay from the log (_NEE_DRT.h:168-230 without the walk): at a null
// collision dL/dsigma = dL/dR . -R / m / (1 - sigma / m); at a real one the
// MIS-weighted dL/dR . (sigma^2 / (1 + sigma^2)) R / sigma (DS: none,
// vr_path_integrator_NEE_DRTDS.h:178-222), then R loses the vertex's light
// terms (T from its record).  Lanes take paths from the primal's list; the
// next collision and the vertex record load one iteration ahead, as in
// k_ds_replay.
template <bool DS>
__global__ void __launch_bounds__(256, 3) k_drt_replay(DMedium M, PathSrc S, const float* __restrict__ dL, float div,
                                                     DScratch* sc, WaveBw wv) {
    const float EPS = 0.00000001f;
    unsigned long long n_list = *((volatile unsigned long long*)&wv.hdr[8]);
    if (n_list > wv.cap_paths) n_list = wv.cap_paths;
    float3 W = f3(0.0f), R = f3(0.0f), dLdR = f3(0.0f);
    bool alive = false, exhausted = false;
    int bounces = 0;
    uint32_t left = 0;  // collisions of the path still to replay
    float4 xs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
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
                    if (e.y != kUnlogged && e.z > 0u) {  // (a path whose log filled runs on the sequential form)
                        const CollisionRec* ep = wv.evs + e.y;
                        xs = __ldcs(&ep->xs);
                        ln = __ldcs(&ep->link);
                        const float4 a = reinterpret_cast<const float4*>(wv.info + 8 * (uint64_t)e.x)[0];
                        dLdR = ld3(dL + 3 * out_index(S, wv.p_begin + e.x)) / div;
                        R = make_float3(a.x, a.y, a.z);
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
            if (!real) {  // _NEE_DRT.h:182-186
                sigma_bw(M, x, dot(dLdR, -R / m / (1.0f - s / m)), tl);
            } else if (ln.z == kNone) {
                guard(sc, 15);  // a scattering collision without its vertex record
                end = true;
            } else {      // _NEE_DRT.h:187-228
                tl.logb += (uint32_t)sizeof(VertexRec);
                const float mis_Ts = DS ? 0.0f : s * s / (1.0f + s * s);
                const float dL_dsigma = DS ? 0.0f : dot(dLdR, mis_Ts * R / s);
                const float Te = __uint_as_float(r0.x), Ts = __uint_as_float(r0.y);
                const float3 sa = make_float3(r1.x, r1.y, r1.z);
                const float ph_nee = r1.w, ph_sun = r2.w;
                const float3 Le = make_float3(r2.x, r2.y, r2.z);
                W = W * sa;
                R = R - W * Te * Le * ph_nee;
                if (M.has_sun) R = R - W * Ts * M.sun_L * ph_sun;
                if (!DS) sigma_bw(M, x, dL_dsigma, tl);
                ++bounces;
                if (all_less(W, EPS) || (M.max_bounces > 0 && bounces >= M.max_bounces)) end = true;
            }
            xs = nxs;
            ln = nln;
            if (--left == 0u) end = true;
            if (end) alive = false;
        }
    }
    flush_counters(sc, VRT_K_DRT_REPLAY, 0, 0, tl);
}

// Host: rounds of primal, light-ray T, their adjoints, replay and reservoir
// branch until every path has been taken; then the handed-over paths on the
// sequential form.
int launch_wave_drt_bw(vrt_context* ctx, const DMedium& M, int bw_mode, const PathSrc& src, uint64_t n_paths,
                       uint64_t seed, const float* dL, float div, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.max_bounces < 0 || M.max_bounces > 4096 || M.tr_mode > 1) return VRT_E_UNSUPPORTED;
    if (bw_mode != VRT_BW_NEE_DRT && bw_mode != VRT_BW_NEE_DRTDS && bw_mode != VRT_BW_NEE_DRTQ)
        return VRT_E_INVALID_ARGUMENT;
    const bool ds = bw_mode == VRT_BW_NEE_DRTDS, q = bw_mode == VRT_BW_NEE_DRTQ;
    if (q && n_paths >= (1ull << 40)) return VRT_E_UNSUPPORTED;  // segment streams take path ids below 2^40
    const unsigned long long lights = M.has_sun ? 2ull : 1ull;
    // uncapped paths (the reference's default) walk at most kUncappedPass
    // vertices here; the few that go on run whole on the sequential form
    const int kpass = M.max_bounces > 0 ? 0 : kUncappedPass;
    const unsigned long long B = (unsigned long long)(M.max_bounces > 0 ? M.max_bounces : kpass);
    int blocksA = persistent_blocks(q ? (const void*)k_drt_primal<true> : (const void*)k_drt_primal<false>, 256,
                                    ctx->num_sms);
    int blocksC = persistent_blocks(ds ? (const void*)k_drt_replay<true> : (const void*)k_drt_replay<false>, 256,
                                    ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocksA > need) blocksA = (int)need;
    if ((uint64_t)blocksC > need) blocksC = (int)need;
    WaveBw wv{};
    wv.lanes = (unsigned long long)blocksA * 256ull;
    const unsigned long long inflight = wv.lanes < n_paths ? wv.lanes : n_paths;
    wv.res_jobs = inflight * (lights * B + 1ull);  // the vertices' light rays and the primary ray's adjoint
    wv.res_recs = inflight * (B + 1);              // B records and the reserved slot after the last one
    wv.cap_jobs = wv.res_jobs + batch_jobs(n_paths, 3ull * lights + 1ull, ctx->batch_limit);
    wv.cap_recs = wv.res_recs + batch_jobs(n_paths, 3, ctx->batch_limit);
    if (wv.cap_recs > (1ull << 30)) return VRT_E_UNSUPPORTED;  // record indices are 30-bit in a job
    wv.cap_paths = (n_paths < (1ull << 24) ? n_paths : (1ull << 24)) + wv.lanes;
    wv.cap_evs = ctx->log_limit ? ctx->log_limit : 4ull * batch_jobs(n_paths, 1, ctx->batch_limit) + inflight * 16ull;
    if (wv.cap_evs > 0xfff00000ull) wv.cap_evs = 0xfff00000ull;  // 32-bit links, kNone / kUnlogged reserved
    wv.res_evs = inflight * 16ull < wv.cap_evs / 2 ? inflight * 16ull : wv.cap_evs / 2;
    wv.kpass = kpass;
    wv.cap_spill = (unsigned long long)n_paths;
    const size_t o_jobs = 256, o_recs = o_jobs + wv.cap_jobs * sizeof(ShadowJob);
    const size_t o_info = o_recs + wv.cap_recs * sizeof(VertexRec), o_resv = o_info + wv.cap_paths * 32;
    const size_t o_list = o_resv + wv.cap_paths * 64;
    const size_t o_evs = o_list + ((wv.cap_paths * 16 + 255) & ~(size_t)255);
    const size_t o_spill = o_evs + wv.cap_evs * 32, o_items = o_spill + ((wv.cap_spill * 8 + 255) & ~(size_t)255);
    // DRTQ: the segments after scattering vertices (at most one per vertex record)
    wv.cap_segs = q ? wv.cap_recs : 0;
    // the branches' items (DRT, DRTDS: one per path; DRTQ: one per segment), their
    // scatter data and the nested paths' estimates
    const unsigned long long cap_items = wv.cap_paths + wv.cap_segs;
    const size_t o_post = o_items + cap_items * 48, o_bR = o_post + cap_items * 48;
    const size_t o_segs = o_bR + ((cap_items * 12 + 255) & ~(size_t)255);
    const size_t bytes = o_segs + wv.cap_segs * 48;
    int st = ensure_wave_buffer(ctx, bytes);
    if (st) return st;
    char* base = static_cast<char*>(ctx->wave);
    wv.hdr = reinterpret_cast<unsigned long long*>(base);
    wv.jobs = reinterpret_cast<ShadowJob*>(base + o_jobs);
    wv.recs = reinterpret_cast<VertexRec*>(base + o_recs);
    wv.info = reinterpret_cast<float*>(base + o_info);
    wv.resv = reinterpret_cast<float4*>(base + o_resv);
    float4* b_items = reinterpret_cast<float4*>(base + o_items);
    float4* b_post = reinterpret_cast<float4*>(base + o_post);
    float* b_R = reinterpret_cast<float*>(base + o_bR);
    wv.segs = q ? reinterpret_cast<float4*>(base + o_segs) : nullptr;
    wv.over = nullptr;
    wv.list = reinterpret_cast<uint4*>(base + o_list);
    wv.evs = reinterpret_cast<CollisionRec*>(base + o_evs);
    wv.spill = reinterpret_cast<unsigned long long*>(base + o_spill);
    wv.spill_count = &wv.hdr[10];  // kept across rounds
    wv.p_begin = 0;
    cudaError_t e = cudaMemsetAsync(&ctx->scratch->next_path, 0, sizeof(unsigned long long), stream);
    if (e != cudaSuccess) return launch_status(e);
    if ((e = cudaMemsetAsync(wv.spill_count, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
        return launch_status(e);
    for (int round = 0;; ++round) {
        // [0] jobs, [1] records, [3] / [4] heads of the shadow kernels, [5] collisions,
        // [7] replay-list head, [8] replay list
        if ((e = cudaMemsetAsync(wv.hdr, 0, 9 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        // [14] DRTQ's segment count
        if (q && (e = cudaMemsetAsync(&wv.hdr[14], 0, sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        {
            KernelScope ks(VRT_K_DRT_PRIMAL, stream);
            if (q) k_drt_primal<true><<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
            else k_drt_primal<false><<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
        }
        count_launches(1);
        if ((st = launch_shadow_record(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream))) return st;
        if ((st = launch_shadow_adjoint(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream, ADJ_DRT)))
            return st;
        {
            KernelScope ks(VRT_K_DRT_REPLAY, stream);
            if (ds) k_drt_replay<true><<<blocksC, 256, 0, stream>>>(M, src, dL, div, ctx->scratch, wv);
            else k_drt_replay<false><<<blocksC, 256, 0, stream>>>(M, src, dL, div, ctx->scratch, wv);
        }
        count_launches(1);
        if ((st = launch_status(cudaGetLastError()))) return st;
        if ((st = launch_drt_branch(M, ds ? 1 : (q ? 2 : 0), src, n_paths, wv.p_begin, &ctx->scratch->next_path,
                                    seed, dL, div, wv.info, wv.resv, wv.cap_paths, wv.segs, &wv.hdr[14], wv.cap_segs,
                                    b_items, b_post, b_R, &wv.hdr[12], ctx->scratch, ctx->num_sms, stream)))
            return st;
        unsigned long long taken = 0;
        if ((e = cudaMemcpyAsync(&taken, &ctx->scratch->next_path, sizeof(taken), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess)
            return launch_status(e);
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
        if (taken >= n_paths) break;
        wv.p_begin = taken;
        if (round > (1 << 20)) return VRT_E_ITER_CAP;
    }
    unsigned long long spilled = 0;
    if ((e = cudaMemcpyAsync(&spilled, wv.spill_count, sizeof(spilled), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return launch_status(e);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
    if (spilled > wv.cap_spill) spilled = wv.cap_spill;
    if (spilled)  // the paths the log could not hold, whole, on the sequential form
        return launch_radiance_bw(M, bw_mode, src, spilled, seed, dL, div, ctx->scratch, ctx->num_sms, stream,
                                  wv.spill);
    return 0;
}

}  // namespace vrt
