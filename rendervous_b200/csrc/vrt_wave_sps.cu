// vrt_wave_sps.cu -- the SPS adjoint as a wavefront (sm_100a).
//
// The reference's singular-path-sampling adjoint
// (include/vr_path_integrator_NEE_SPS.h:104-263) walks each path twice with
// the same draws: the primal (collision positions by delta tracking against
// majorant + 1e-6, while MIS is allowed a choice between that position and a
// uniform point of the segment -- the singular vertex, after which the light
// terms go to Rf and are weighed by its sigma), then the replay (at every
// vertex a sigma scatter, a stratified scatter of dL/dtau over the segment on
// the second stream, the light rays' transmittance adjoints).  The replay
// changes nothing on the path, so the primal logs what it recomputes:
//
//   k_sps_primal   per vertex a 32-byte segment record (position, sigma,
//                  weight; the segment's sample count, the singular and MIS
//                  flags) and a vertex record; a job per light (record word
//                  bit 1: after the singular vertex); per path its entry point
//                  and the singular vertex's sigma; the primary ray's
//                  environment adjoint as an adjoint-only job
//   (vrt_wave.cu)  T of every job into its record and R / Rf; the jobs'
//                  adjoints from fork j of stream 1, weighed by the singular
//                  sigma after the singular vertex
//   k_sps_replay   the sigma scatters and the stratified dL/dtau scatters,
//                  the latter drawing stream 1's uniforms in path order (the
//                  forks the adjoints take do not move that stream's counter)
//
// Compiled with -fmad=false like the sequential form (vrt_path.cu).  Paths the
// log cannot hold, and uncapped paths still going after kUncappedPass
// vertices, run whole on the sequential form afterwards, over a list of their
// ids (their jobs here are skipped: first-collision word kSpilled).
#include "vrt_wave.cuh"

namespace vrt {

using namespace wave;

namespace {

__device__ __forceinline__ float3 ray_at(float3 x, float3 w, float t) {
    return make_float3(__fadd_rn(x.x, __fmul_rn(w.x, t)), __fadd_rn(x.y, __fmul_rn(w.y, t)),
                       __fadd_rn(x.z, __fmul_rn(w.z, t)));
}

// vr_path_integrator_NEE_SPS.h:1-59 sample_collision_position, the
// sequential form's arithmetic (pow(sigma, 3) as sigma * sigma * sigma);
// returns whether the uniform point was taken (the singular vertex).
__device__ __forceinline__ bool sps_collision(const DMedium& M, Rng& rng, float3 x, float3 w, float d, float3& xc,
                                              float& weight_xc, float& sigma_xc, int& samples, bool& mis_allowed,
                                              Tally& tl, DScratch* sc) {
    float t = 0.0f;
    weight_xc = 0.0f;
    sigma_xc = 0.0f;
    samples = 0;
    xc = x;
    int it = 0;
    for (; it < kStepCap; ++it) {
        float md;
        const float m = majorant(M, xc, w, md) + 0.000001f;
        const float dt = gmin(-logf(1.0f - rng.uniform()) / m, gmin(md, d - t));
        t += dt;
        xc = ray_at(x, w, t);
        ++tl.steps;
        if (dt >= md - 0.0000001f) continue;
        if (t >= d - 0.0000001f) break;
        const float s = sigma(M, xc, tl);
        samples++;
        if (rng.uniform() < s / m) {
            weight_xc = 1.0f;
            sigma_xc = s;
            break;
        }
    }
    if (it == kStepCap) raise_status(&sc->status, 4);
    if (!mis_allowed) return false;
    const float powered_c = sigma_xc * sigma_xc * sigma_xc;
    const float mis_wc = weight_xc * powered_c / (1.0f + powered_c);
    const float u = rng.uniform();
    const float3 xf = xc * (1.0f - u) + x * u;
    const float sigma_f = sigma(M, xf, tl);
    const float powered_f = sigma_f * sigma_f * sigma_f;
    const float mis_wf = t / (1.0f + powered_f);
    weight_xc = mis_wc + mis_wf;
    if (rng.uniform() * weight_xc < mis_wf) {
        xc = xf;
        sigma_xc = sigma_f;
        mis_allowed = false;
        return true;
    }
    return false;
}

}  // namespace

__global__ void __launch_bounds__(256, 3) k_sps_primal(DMedium M, PathSrc S, uint64_t n_paths, uint64_t seed,
                                                     DScratch* sc, WaveBw wv) {
    const unsigned lane = threadIdx.x & 31u;
    const float EPS = 0.00001f;  // _NEE_SPS.h:121
    const int lights = M.has_sun ? 2 : 1;
    Rng rng;
    float3 x = f3(0.0f), w = f3(0.0f), W = f3(0.0f);
    float d = 0.0f, W_singular = 1.0f;
    bool alive = false, exhausted = false, logged = false, mis_allowed = true;
    int bounces = 0;
    uint64_t pid = 0;
    uint32_t first = kNone, rec_next = kNone, first_ev = kNone, ev_next = kNone, n_ev = 0;
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
                    ++n_paths_done;
                    __stcs(wv.resv + k, make_float4(x.x, x.y, x.z, 1.0f));  // entry point, singular sigma
                    if (!(d > 0.0f)) {  // _NEE_SPS.h:110: nothing to do
                        put_job(wv.jobs, jb + rank, x, w, f3(0.0f), job_key(pid, 0), kAdjOnly);
                        float* io = wv.info + 8 * k;
                        __stcs(reinterpret_cast<float4*>(io), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
                        __stcs(reinterpret_cast<float4*>(io) + 1,
                               make_float4(0.0f, 0.0f, __uint_as_float(kNone), __uint_as_float(kNone)));
                    } else {
                        // _NEE_SPS.h:115-116: the primal's T of the primary ray takes fork 0 of the
                        // path's stream (unused); its adjoint, fork 0 of stream 1
                        rng.ntr += 1u;
                        put_job(wv.jobs, jb + rank, x, w, env_radiance(M, w), job_key(pid, 0), kAdjOnly);
                        W = f3(1.0f);
                        W_singular = 1.0f;
                        mis_allowed = true;
                        bounces = 0;
                        first = kNone;
                        rec_next = kNone;
                        first_ev = kNone;
                        ev_next = kNone;
                        n_ev = 0;
                        logged = true;
                        alive = true;
                    }
                }
            }
        }
        if (__all_sync(kAll, !alive && exhausted)) break;

        int nrec = 0, nj = 0, nev = 0;
        bool finish = false, spill = false, after = true;
        float3 xc = f3(0.0f), wnee = f3(0.0f), sa = f3(0.0f), Le = f3(0.0f);
        float weight_xc = 0.0f, sigma_xc = 0.0f, ph_env = 0.0f, ph_sun = 0.0f;
        uint32_t jfork = 0, flags = 0;
        if (alive) {  // one vertex per iteration (_NEE_SPS.h:123-145)
            int samples = 0;
            const bool singular =
                sps_collision(M, rng, x, w, d, xc, weight_xc, sigma_xc, samples, mis_allowed, tl, sc);
            if (singular) W_singular = sigma_xc;
            if (weight_xc == 0.0f) {
                finish = true;
            } else {
                after = mis_allowed;
                flags = (singular ? 1u : 0u) | (mis_allowed ? 2u : 0u) | ((uint32_t)samples << 2);
                x = xc;
                sa = albedo(M, x, tl);
                W = W * (weight_xc * sa);
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
                nrec = rec_next == kNone ? 2 : 1;
                nev = logged ? (ev_next == kNone ? 2 : 1) : 0;
                nj = lights;
                if (all_less(W, EPS) || capped) {
                    finish = true;
                } else if (wv.kpass > 0 && bounces >= wv.kpass) {
                    finish = true;  // an uncapped path past the pass budget: whole, on the sequential form
                    spill = true;
                }
            }
        }
        // ---- one reservation for the light jobs, the vertex record, the segment
        // record and (at the end of a path with logged vertices) its replay-list entry
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
        if (nev) {  // the segment record, with the slot of the path's next one
            const unsigned long long je = ev_next == kNone ? sl.s2 : ev_next;
            const unsigned long long jn = ev_next == kNone ? sl.s2 + 1 : sl.s2;
            if (je >= wv.cap_evs || jn >= wv.cap_evs) {
                logged = false;  // the log is full: the path runs whole on the sequential form
                finish = true;
                spill = true;
            } else {
                CollisionRec* ep = wv.evs + je;
                __stcs(&ep->xs, make_float4(x.x, x.y, x.z, sigma_xc));
                __stcs(&ep->link, make_uint4(__float_as_uint(weight_xc), (uint32_t)jn, (uint32_t)r, flags));
                tl.logb += (uint32_t)sizeof(CollisionRec);
                if (first_ev == kNone) first_ev = (uint32_t)je;
                ev_next = (uint32_t)jn;
                ++n_ev;
            }
        }
        if (nj) {  // the light rays of the vertex, weighed W * L * phase; bit 1: after the singular vertex
            const unsigned long long j = sl.s0;
            const uint32_t tgt = ((uint32_t)r << 2) | (after ? 0u : 2u);
            put_job(wv.jobs, j, x, wnee, W * Le * ph_env, job_key(pid, jfork), tgt);
            if (nj == 2) put_job(wv.jobs, j + 1, x, M.sun_dir, W * M.sun_L * ph_sun, job_key(pid, jfork + 1), tgt | 1u);
        }
        if (finish) {  // the path's words: R and Rf (filled by the light rays), first record and segment
            const uint64_t k = pid - wv.p_begin;
            float* io = wv.info + 8 * k;
            __stcs(reinterpret_cast<float4*>(io), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
            __stcs(reinterpret_cast<float4*>(io) + 1,
                   make_float4(0.0f, 0.0f, __uint_as_float(first), __uint_as_float(spill ? kSpilled : first_ev)));
            if (nl) __stcs(wv.list + sl.s3, make_uint4((uint32_t)k, logged ? first_ev : kUnlogged, n_ev, 0u));
            reinterpret_cast<float*>(wv.resv + k)[3] = W_singular;
            if (spill) {
                const unsigned long long o = atomicAdd(wv.spill_count, 1ull);
                if (o < wv.cap_spill) wv.spill[o] = (unsigned long long)pid;
                else guard(sc, 14);
            }
            alive = false;
        }
    }
    flush_counters(sc, VRT_K_SPS_PRIMAL, n_paths_done, 0, tl);
}

// The SPS replay from the log (_NEE_SPS.h:203-261 without the walk): per
// vertex dL/dsigma (the singular vertex: dL/dR . Rf; else dL/dR . (R + W_s Rf)
// / max(0.001, sigma)) and dL/dtau = -dL/dR . (R + W_s Rf) spread over the
// segment in max(samples, 1) stratified bins from stream 1; then R (before the
// singular vertex) or Rf loses the vertex's light terms (T from its record).
// Lanes take paths from the primal's list; the next segment and the vertex
// record load one iteration ahead.
__global__ void __launch_bounds__(256, 3) k_sps_replay(DMedium M, PathSrc S, uint64_t seed, const float* __restrict__ dL,
                                                     float div, DScratch* sc, WaveBw wv) {
    const float EPS = 0.00001f;
    unsigned long long n_list = *((volatile unsigned long long*)&wv.hdr[8]);
    if (n_list > wv.cap_paths) n_list = wv.cap_paths;
    float3 W = f3(0.0f), R = f3(0.0f), Rf = f3(0.0f), dLdR = f3(0.0f), prev = f3(0.0f);
    float W_singular = 1.0f;
    Rng sec;  // stream 1: the stratified bins' uniforms, in path order
    bool alive = false, exhausted = false;
    int bounces = 0;
    uint32_t left = 0;
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
                    if (e.y != kUnlogged && e.z > 0u) {
                        const CollisionRec* ep = wv.evs + e.y;
                        xs = __ldcs(&ep->xs);
                        ln = __ldcs(&ep->link);
                        const float4* io = reinterpret_cast<const float4*>(wv.info + 8 * (uint64_t)e.x);
                        const float4 a = io[0], b = io[1];
                        const float4 ent = wv.resv[e.x];
                        const uint64_t pid = wv.p_begin + e.x;
                        dLdR = ld3(dL + 3 * out_index(S, pid)) / div;
                        R = make_float3(a.x, a.y, a.z);
                        Rf = make_float3(a.w, b.x, b.y);
                        prev = make_float3(ent.x, ent.y, ent.z);
                        W_singular = ent.w;
                        sec.init(seed, pid, 1u);
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
            float4 nxs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            uint4 nln = make_uint4(0u, kNone, kNone, 0u);
            if (left > 1u) {
                const CollisionRec* np = wv.evs + ln.y;
                nxs = __ldcs(&np->xs);
                nln = __ldcs(&np->link);
            }
            tl.logb += (uint32_t)(sizeof(CollisionRec) + sizeof(VertexRec));
            const uint4* rp = reinterpret_cast<const uint4*>(wv.recs + ln.z);
            const uint4 r0 = __ldcs(rp);
            const float4 r1 = __ldcs(reinterpret_cast<const float4*>(rp + 1));
            const float4 r2 = __ldcs(reinterpret_cast<const float4*>(rp + 2));
            const float3 x = make_float3(xs.x, xs.y, xs.z);
            const float sigma_xc = xs.w, weight_xc = __uint_as_float(ln.x);
            const bool singular = (ln.w & 1u) != 0u, mis_allowed = (ln.w & 2u) != 0u;
            const int samples = (int)(ln.w >> 2);
            const float3 further_R = R + W_singular * Rf;
            const float k = dot(dLdR, further_R);
            const float dL_dtau = -k;
            const float dL_dsigma = singular ? dot(dLdR, Rf) : k / gmax(0.001f, sigma_xc);
            W = W * weight_xc;
            W = W * make_float3(r1.x, r1.y, r1.z);
            const float Te = __uint_as_float(r0.x), Ts = __uint_as_float(r0.y);
            const float ph_nee = r1.w, ph_sun = r2.w;
            const float3 Le = make_float3(r2.x, r2.y, r2.z);
            float3 added_R = W * Te * ph_nee * Le;
            if (M.has_sun) added_R = added_R + W * Ts * ph_sun * M.sun_L;
            if (mis_allowed) R = R - added_R;
            else Rf = Rf - added_R;
            sigma_bw(M, x, dL_dsigma, tl);
            // st_tau_bw (_NEE_SPS.h:88-101): stratified bins over the segment prev -> x
            const int bins = samples > 1 ? samples : 1;
            if (dL_dtau != 0.0f) {
                const float dd = sqrtf(dot(x - prev, x - prev));
                const float g = dL_dtau * dd / (float)bins;
                for (int i = 0; i < bins; ++i) {
                    const float f = ((float)i + sec.uniform()) / (float)bins;
                    sigma_bw(M, prev * (1.0f - f) + x * f, g, tl);
                }
            }
            ++tl.steps;
            ++bounces;
            if (all_less(W, EPS) || (M.max_bounces > 0 && bounces >= M.max_bounces)) end = true;
            prev = x;
            xs = nxs;
            ln = nln;
            if (--left == 0u) end = true;
            if (end) alive = false;
        }
    }
    flush_counters(sc, VRT_K_SPS_REPLAY, 0, 0, tl);
}

// Host: rounds of primal, light-ray T, their adjoints and replay until every
// path has been taken; then the handed-over paths on the sequential form.
int launch_wave_sps_bw(vrt_context* ctx, const DMedium& M, const PathSrc& src, uint64_t n_paths, uint64_t seed,
                       const float* dL, float div, cudaStream_t stream) {
    if (n_paths == 0) return 0;
    if (M.max_bounces < 0 || M.max_bounces > 4096 || M.tr_mode > 1) return VRT_E_UNSUPPORTED;
    const unsigned long long lights = M.has_sun ? 2ull : 1ull;
    const int kpass = M.max_bounces > 0 ? 0 : kUncappedPass;
    const unsigned long long B = (unsigned long long)(M.max_bounces > 0 ? M.max_bounces : kpass);
    int blocksA = persistent_blocks((const void*)k_sps_primal, 256, ctx->num_sms);
    int blocksC = persistent_blocks((const void*)k_sps_replay, 256, ctx->num_sms);
    const uint64_t need = (n_paths + 255) / 256;
    if ((uint64_t)blocksA > need) blocksA = (int)need;
    if ((uint64_t)blocksC > need) blocksC = (int)need;
    WaveBw wv{};
    wv.lanes = (unsigned long long)blocksA * 256ull;
    const unsigned long long inflight = wv.lanes < n_paths ? wv.lanes : n_paths;
    wv.res_jobs = inflight * (lights * B + 1ull);  // the vertices' light rays and the primary ray's adjoint
    wv.res_recs = inflight * (B + 1);
    wv.cap_jobs = wv.res_jobs + batch_jobs(n_paths, 3ull * lights + 1ull, ctx->batch_limit);
    wv.cap_recs = wv.res_recs + batch_jobs(n_paths, 3, ctx->batch_limit);
    if (wv.cap_recs > (1ull << 30)) return VRT_E_UNSUPPORTED;  // record indices are 30-bit in a job
    wv.cap_paths = (n_paths < (1ull << 24) ? n_paths : (1ull << 24)) + wv.lanes;
    // one segment record per vertex
    wv.cap_evs = ctx->log_limit ? ctx->log_limit : wv.cap_recs;
    if (wv.cap_evs > 0xfff00000ull) wv.cap_evs = 0xfff00000ull;  // 32-bit links, kNone / kUnlogged reserved
    wv.res_evs = wv.res_recs < wv.cap_evs / 2 ? wv.res_recs : wv.cap_evs / 2;
    wv.kpass = kpass;
    wv.cap_spill = (unsigned long long)n_paths;
    const size_t o_jobs = 256, o_recs = o_jobs + wv.cap_jobs * sizeof(ShadowJob);
    const size_t o_info = o_recs + wv.cap_recs * sizeof(VertexRec), o_resv = o_info + wv.cap_paths * 32;
    const size_t o_list = o_resv + wv.cap_paths * 16;
    const size_t o_evs = o_list + ((wv.cap_paths * 16 + 255) & ~(size_t)255);
    const size_t o_spill = o_evs + wv.cap_evs * 32, bytes = o_spill + wv.cap_spill * 8;
    int st = ensure_wave_buffer(ctx, bytes);
    if (st) return st;
    char* base = static_cast<char*>(ctx->wave);
    wv.hdr = reinterpret_cast<unsigned long long*>(base);
    wv.jobs = reinterpret_cast<ShadowJob*>(base + o_jobs);
    wv.recs = reinterpret_cast<VertexRec*>(base + o_recs);
    wv.info = reinterpret_cast<float*>(base + o_info);
    wv.resv = reinterpret_cast<float4*>(base + o_resv);
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
        // [0] jobs, [1] records, [3] / [4] heads of the shadow kernels, [5] segments,
        // [7] replay-list head, [8] replay list
        if ((e = cudaMemsetAsync(wv.hdr, 0, 9 * sizeof(unsigned long long), stream)) != cudaSuccess)
            return launch_status(e);
        {
            KernelScope ks(VRT_K_SPS_PRIMAL, stream);
            k_sps_primal<<<blocksA, 256, 0, stream>>>(M, src, n_paths, seed, ctx->scratch, wv);
        }
        count_launches(1);
        if ((st = launch_shadow_record(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream))) return st;
        if ((st = launch_shadow_adjoint(M, src, wv, seed, dL, div, ctx->scratch, ctx->num_sms, stream, ADJ_SPS)))
            return st;
        {
            KernelScope ks(VRT_K_SPS_REPLAY, stream);
            k_sps_replay<<<blocksC, 256, 0, stream>>>(M, src, seed, dL, div, ctx->scratch, wv);
        }
        count_launches(1);
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
    unsigned long long spilled = 0;
    if ((e = cudaMemcpyAsync(&spilled, wv.spill_count, sizeof(spilled), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return launch_status(e);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return launch_status(e);
    if (spilled > wv.cap_spill) spilled = wv.cap_spill;
    if (spilled)  // the paths the log could not hold and the long uncapped ones, whole, on the sequential form
        return launch_radiance_bw(M, VRT_BW_NEE_SPS, src, spilled, seed, dL, div, ctx->scratch, ctx->num_sms, stream,
                                  wv.spill);
    return 0;
}

}  // namespace vrt
