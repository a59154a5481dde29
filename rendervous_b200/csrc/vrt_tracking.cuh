// vrt_tracking.cuh -- transmittance estimators along one ray (sm_100a).
//
//   DDA   include/vr_transmittance_DDA.h:1-156 (midpoint rule of the reference,
//         or the exact per-cell integral: two-point Gauss-Legendre is exact for
//         the cubic a trilinear field becomes on a segment)
//   RT    include/vr_transmittance_RT.h:1-141 (ratio tracking, RR at 0.01 / 0.1)
//   DT    include/vr_transmittance_DT.h:1-90  (delta tracking)
//   GRT / GDT  include/vr_transmittance_GRT.h:1-83, _GDT.h:1-84 (ratio / delta
//         tracking of the residual over per-cell minorants, on the DDA walk)
//
// The DDA keeps the 8 corner values of the current cell in registers: a step
// along axis a keeps the face the ray crosses into and loads only the 4 new
// corners (the reference reloads all 8; the values are identical because the
// clamped node indices coincide).  Its adjoint likewise carries the gradient
// of the shared face and issues 4 atomic adds per cell instead of 8.
#pragma once
#include "vrt_device.cuh"

namespace vrt {

constexpr int kStepCap = 1 << 24;  // per-segment iteration bound (error VRT_E_ITER_CAP)

// Optical distance of the current free flight.  With a piecewise-constant
// majorant a flight continues across a majorant-brick face with the optical
// depth it has left (exponential lengths are memoryless), so a draw is taken
// only after the previous flight ended at a candidate collision or at the end
// of the segment.  The constant majorant (distance 1e6) never crosses a face,
// so then every step draws, as the reference does.
// Majorant bricks along one straight segment (majorant-grid mode): a 3D DDA
// over the brick grid, started at the segment's first query.  The brick of the
// start point gets the 1e-4-brick nudge of majorant(), face distances use
// correctly rounded reciprocals, and outside the grid's box the bound is 0.
// Inert with the constant majorant.  Axis selection is by branches so the
// state stays in registers.  Whether the segment reaches the grid at all is
// tested once, at the start (a segment that does not gets no face: infinite
// face distances); one that leaves the grid walks on through bound-0 bricks
// until it ends, so a query tests nothing but the three face distances.
struct BrickWalk {
    bool live = false;
    int c0, c1, c2, s0, s1, s2;
    float n0, n1, n2, d0, d1, d2, t, m;

    __device__ __forceinline__ void reset() { live = false; }
    __device__ __forceinline__ float lookup(const DMedium& M) const {
        if ((unsigned)c0 >= (unsigned)M.Mx || (unsigned)c1 >= (unsigned)M.My || (unsigned)c2 >= (unsigned)M.Mz)
            return 0.0f;
        return __ldg(M.maj + ((c2 * M.My + c1) * M.Mx + c0));
    }
    __device__ __forceinline__ static void axis_init(float x, float bmin, float scale, float w, int& c, int& st, float& n,
                                                     float& dd) {
        const float inf = __int_as_float(0x7f800000);
        float q = (x - bmin) * scale;
        float dq = w * scale;
        if (dq > 0.0f) {
            c = (int)floorf(q + 1e-4f); st = 1;
            float rv = __frcp_rn(dq);
            n = ((float)(c + 1) - q) * rv; dd = rv;
        } else if (dq < 0.0f) {
            c = (int)floorf(q - 1e-4f); st = -1;
            float rv = __frcp_rn(dq);
            n = ((float)c - q) * rv; dd = -rv;
        } else {
            c = (int)floorf(q); st = 0; n = inf; dd = inf;
        }
    }
    __device__ __forceinline__ void init(const DMedium& M, float3 x, float3 w) {
        live = true;
        t = 0.0f;
        axis_init(x.x, M.bmin.x, M.maj_scale.x, w.x, c0, s0, n0, d0);
        axis_init(x.y, M.bmin.y, M.maj_scale.y, w.y, c1, s1, n1, d1);
        axis_init(x.z, M.bmin.z, M.maj_scale.z, w.z, c2, s2, n2, d2);
        m = lookup(M);
        if (never_enters(M)) {  // a segment that never reaches the grid: no face to cross
            const float inf = __int_as_float(0x7f800000);
            n0 = inf; n1 = inf; n2 = inf;
        }
    }
    __device__ __forceinline__ bool never_enters(const DMedium& M) const {
        return (c0 < 0 && s0 <= 0) || (c0 >= M.Mx && s0 >= 0) || (c1 < 0 && s1 <= 0) || (c1 >= M.My && s1 >= 0) ||
               (c2 < 0 && s2 <= 0) || (c2 >= M.Mz && s2 >= 0);
    }
    // (majorant, distance to the next brick face) at the walk's position
    __device__ __forceinline__ float query(const DMedium& M, float3 x, float3 w, float& md) {
        if (M.maj_mode == 0) { md = 1000000.0f; return M.gmaj; }
        if (!live) init(M, x, w);
        float nt = (n0 <= n1 && n0 <= n2) ? n0 : (n1 <= n2 ? n1 : n2);
        md = nt - t;
        return m;
    }
    __device__ __forceinline__ void advance(const DMedium& M) {
        if (!live) return;
        if (n0 <= n1 && n0 <= n2) { t = n0; n0 += d0; c0 += s0; }
        else if (n1 <= n2) { t = n1; n1 += d1; c1 += s1; }
        else { t = n2; n2 += d2; c2 += s2; }
        m = lookup(M);
    }
    __device__ __forceinline__ void move(float dist) { t += dist; }
};

struct Flight {
    float tau = -1.0f;
    int it = 0;
    BrickWalk bk;  // majorant bricks of the current segment
    __device__ __forceinline__ float sample(Rng& rng) {
        if (tau < 0.0f) tau = -logf(1.0f - rng.uniform());
        return tau;
    }
    __device__ __forceinline__ void cross(float m, float md) { tau -= __fmul_rn(m, md); }
    __device__ __forceinline__ void used() { tau = -1.0f; }
};

struct DDA {
    float3 x, w, alpha, alpha_inc, vn, vm;
    int cx, cy, cz, sx, sy, sz, dimx, dimy, dimz;
    float d;
    float s[8];  // corner values, index dz*4 + dy*2 + dx

    // vr_transmittance_DDA.h:3-36.  false when the ray misses (T = 1).
    __device__ __forceinline__ bool init(const DMedium& M, float3 x0, float3 w0) {
        float tMin, tMax;
        if (!boundary(M, x0, w0, tMin, tMax)) return false;
        float gMin, gMax;
        if (!intersect_ray_box(x0, w0, M.bmin, M.bmax, gMin, gMax)) return false;
        tMin = gmax(tMin, gMin);
        tMax = gmin(tMax, gMax);
        if (tMax <= tMin) return false;
        w = w0;
        x = x0 + w0 * tMin;
        d = tMax - tMin;
        dimx = M.sigma.W - 1; dimy = M.sigma.H - 1; dimz = M.sigma.D - 1;
        float3 fdim = make_float3((float)dimx, (float)dimy, (float)dimz);
        float3 box_size = M.bmax - M.bmin;
        float3 cell_size = box_size / fdim;
        float3 den = make_float3(gmax(0.000001f, fabsf(w.x)), gmax(0.000001f, fabsf(w.y)), gmax(0.000001f, fabsf(w.z)));
        alpha_inc = cell_size / den;
        sx = w.x > 0.0f ? 1 : (w.x < 0.0f ? -1 : 0);
        sy = w.y > 0.0f ? 1 : (w.y < 0.0f ? -1 : 0);
        sz = w.z > 0.0f ? 1 : (w.z < 0.0f ? -1 : 0);
        vn = (x - M.bmin) * fdim / box_size;
        vm = w * fdim / box_size;
        reset(M);
        return true;
    }
    // cell and alpha at the start of the segment (also used to replay it)
    __device__ __forceinline__ void reset(const DMedium& M) {
        float3 fdim = make_float3((float)dimx, (float)dimy, (float)dimz);
        float3 box_size = M.bmax - M.bmin;
        float3 cell_size = box_size / fdim;
        cx = min(max((int)vn.x, 0), dimx - 1);
        cy = min(max((int)vn.y, 0), dimy - 1);
        cz = min(max((int)vn.z, 0), dimz - 1);
        float3 corner = (make_float3((float)cx, (float)cy, (float)cz) + make_float3((float)sx, (float)sy, (float)sz) * 0.5f +
                         f3(0.5f)) * cell_size + M.bmin;
        float3 den = make_float3(gmax(0.000001f, fabsf(w.x)), gmax(0.000001f, fabsf(w.y)), gmax(0.000001f, fabsf(w.z)));
        float3 cd = corner - x;
        alpha = make_float3(fabsf(cd.x), fabsf(cd.y), fabsf(cd.z)) / den;
    }
    // vr_sigma_grid.h:1-7 sigma_at: node clamped to [0, dim]
    __device__ __forceinline__ int node(const DGrid& g, int x_, int y_, int z_) const {
        x_ = min(max(x_, 0), dimx); y_ = min(max(y_, 0), dimy); z_ = min(max(z_, 0), dimz);
        return z_ * g.sD + y_ * g.sH + x_ * g.sW;
    }
    __device__ __forceinline__ void load_all(const DGrid& g) {
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = ldg(g.data + node(g, cx + (k & 1), cy + ((k >> 1) & 1), cz + (k >> 2)));
    }
    // vr_sigma_grid.h:18-27 interpolated_sigma
    __device__ __forceinline__ float interp(float3 a) const {
        return mixf(mixf(mixf(s[0], s[1], a.x), mixf(s[2], s[3], a.x), a.y),
                    mixf(mixf(s[4], s[5], a.x), mixf(s[6], s[7], a.x), a.y), a.z);
    }
    __device__ __forceinline__ float3 ialpha(float t) const {
        return (vm * t + vn) - make_float3((float)cx, (float)cy, (float)cz);
    }
    // vr_transmittance_DDA.h:48-55: the axis of the next step (0,1,2)
    __device__ __forceinline__ int next_axis() const {
        return (alpha.x <= alpha.y && alpha.x <= alpha.z) ? 0 : ((alpha.x > alpha.y && alpha.y <= alpha.z) ? 1 : 2);
    }
    // one step along `axis` (selects, no branch on the axis)
    __device__ __forceinline__ void step(int axis) {
        alpha.x = axis == 0 ? alpha.x + alpha_inc.x : alpha.x;
        alpha.y = axis == 1 ? alpha.y + alpha_inc.y : alpha.y;
        alpha.z = axis == 2 ? alpha.z + alpha_inc.z : alpha.z;
        cx += axis == 0 ? sx : 0;
        cy += axis == 1 ? sy : 0;
        cz += axis == 2 ? sz : 0;
    }
    // returns the axis stepped
    __device__ __forceinline__ int advance_cell() {
        const int axis = next_axis();
        step(axis);
        return axis;
    }
    // Node offsets of the current cell's corners, clamped as sigma_at clamps
    // (vr_sigma_grid.h:1-7): o[0..1] along x, o[2..3] along y, o[4..5] along z.
    __device__ __forceinline__ void corner_offsets(const DGrid& g, int* o) const {
        o[0] = min(max(cx, 0), dimx) * g.sW;
        o[1] = min(max(cx + 1, 0), dimx) * g.sW;
        o[2] = min(max(cy, 0), dimy) * g.sH;
        o[3] = min(max(cy + 1, 0), dimy) * g.sH;
        o[4] = min(max(cz, 0), dimz) * g.sD;
        o[5] = min(max(cz + 1, 0), dimz) * g.sD;
    }
    // After a step along `axis`: the corners on the face crossed into (slots
    // whose `axis` bit is 1 after a step up, 0 after a step down) load at the
    // new cell; the opposite face takes the values they had.  Selects and
    // predicated loads instead of a branch per axis and sign, so lanes that
    // step along different axes stay converged; every slot gets the value the
    // per-axis form gave it.
    __device__ __forceinline__ void shift_load(const DGrid& g, int axis) {
        const int st = axis == 0 ? sx : (axis == 1 ? sy : sz);
        if (st == 0) return;
        const int m = 1 << axis, far = st > 0 ? m : 0;
        int o[6];
        corner_offsets(g, o);
        float ns[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float v = axis == 0 ? s[k ^ 1] : (axis == 1 ? s[k ^ 2] : s[k ^ 4]);
            if ((k & m) == far) v = ldg(g.data + (o[4 + (k >> 2)] + o[2 + ((k >> 1) & 1)] + o[k & 1]));
            ns[k] = v;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = ns[k];
    }

    static constexpr float kGL = 0.28867513459481288225f;  // 1 / (2 sqrt 3)

    // One cell of tau: its (midpoint or Gauss-Legendre) integral into the
    // compensated (Kahan) sum, then the step and the new face's loads.
    template <bool EXACT>
    __device__ __forceinline__ void tau_cell(const DGrid& g, float& acc, float& comp_err, float& ct) {
        float nt = gmin(d, gmin(alpha.x, gmin(alpha.y, alpha.z)));
        float dt = nt - ct;
        float term;
        if (!EXACT) {
            term = interp(ialpha(mixf(ct, nt, 0.5f))) * dt;
        } else {
            float mid = mixf(ct, nt, 0.5f), h = dt * kGL;
            term = (interp(ialpha(mid - h)) + interp(ialpha(mid + h))) * (dt * 0.5f);
        }
        float yk = term - comp_err;
        float tk = acc + yk;
        comp_err = (tk - acc) - yk;
        acc = tk;
        ct = nt;
        int axis = advance_cell();
        shift_load(g, axis);
    }
    // the reference stops 1e-4 short of the exit (vr_transmittance_DDA.h:38);
    // the exact mode integrates the whole segment
    template <bool EXACT>
    __device__ __forceinline__ float tau_stop() const { return EXACT ? d : d - 0.0001f; }

    // tau over the segment; one step and one (8-corner) lookup per cell
    template <bool EXACT>
    __device__ __forceinline__ float tau(const DGrid& g, Tally& tl) {
        float acc = 0.0f, comp_err = 0.0f, ct = 0.0f;
        load_all(g);
        int it = 0;
        const float stop = tau_stop<EXACT>();
        while (ct < stop && it < kStepCap) {
            tau_cell<EXACT>(g, acc, comp_err, ct);
            ++tl.steps;
            ++tl.lookups;
            ++it;
        }
        return acc;
    }

    // vr_sigma_grid.h:29-39 interpolated_sigma_bw, added into acc[8]
    __device__ __forceinline__ static void add_weights(float3 a, float dL, float* acc) {
        acc[0] += dL * (1.0f - a.x) * (1.0f - a.y) * (1.0f - a.z);
        acc[1] += dL * (a.x) * (1.0f - a.y) * (1.0f - a.z);
        acc[2] += dL * (1.0f - a.x) * (a.y) * (1.0f - a.z);
        acc[3] += dL * (a.x) * (a.y) * (1.0f - a.z);
        acc[4] += dL * (1.0f - a.x) * (1.0f - a.y) * (a.z);
        acc[5] += dL * (a.x) * (1.0f - a.y) * (a.z);
        acc[6] += dL * (1.0f - a.x) * (a.y) * (a.z);
        acc[7] += dL * (a.x) * (a.y) * (a.z);
    }
    __device__ __forceinline__ void flush(const DGrid& g, float* acc, int k) const {
        if (acc[k] != 0.0f) red_add(g.grad + node(g, cx + (k & 1), cy + ((k >> 1) & 1), cz + (k >> 2)), acc[k]);
        acc[k] = 0.0f;
    }
    // Before a step along `axis`: the sums of the face left behind go to the
    // gradient, those of the face crossed into move to the opposite slots
    // (they are that face's corners in the next cell).  Selects and predicated
    // atomics, as in shift_load.
    __device__ __forceinline__ void carry(const DGrid& g, float* acc, int axis) const {
        const int st = axis == 0 ? sx : (axis == 1 ? sy : sz);
        if (st == 0) return;
        const int m = 1 << axis, far = st > 0 ? m : 0;
        int o[6];
        corner_offsets(g, o);
        // after a y or z step the face left behind holds two x-neighbour pairs:
        // one vector atomic each where the nodes are adjacent (red_add2 falls
        // back to two scalar adds where the pair is not 8-byte aligned)
        const bool pairs = axis != 0 && g.sW == 1 && o[1] == o[0] + 1;
        float na[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const bool behind = (k & m) != far;
            float* a = g.grad + (o[4 + (k >> 2)] + o[2 + ((k >> 1) & 1)] + o[k & 1]);
            if (pairs) {
                if (behind && (k & 1) == 0 && (acc[k] != 0.0f || acc[(k + 1) & 7] != 0.0f))
                    red_add2(a, acc[k], acc[(k + 1) & 7]);
            } else if (behind && acc[k] != 0.0f) {
                red_add(a, acc[k]);
            }
            const float v = axis == 0 ? acc[k ^ 1] : (axis == 1 ? acc[k ^ 2] : acc[k ^ 4]);
            na[k] = behind ? v : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = na[k];
    }
    // One cell of the second march (vr_transmittance_DDA.h:121-153): the
    // cell's dL/dsigma per corner into acc, then the step (the face shared with
    // the next cell stays in registers).
    template <bool EXACT>
    __device__ __forceinline__ void scatter_cell(const DGrid& g, float dL_dtau, float* acc, float& ct) {
        float nt = gmin(d, gmin(alpha.x, gmin(alpha.y, alpha.z)));
        float dt = nt - ct;
        if (!EXACT) {
            add_weights(ialpha(mixf(ct, nt, 0.5f)), dL_dtau * dt, acc);
        } else {
            float mid = mixf(ct, nt, 0.5f), h = dt * kGL;
            add_weights(ialpha(mid - h), dL_dtau * dt * 0.5f, acc);
            add_weights(ialpha(mid + h), dL_dtau * dt * 0.5f, acc);
        }
        ct = nt;
        // flush the face left behind, move the crossed face to its new slot
        const int axis = next_axis();
        carry(g, acc, axis);
        step(axis);
    }
    // acc holds the corners of the cell the march stopped in (the face
    // carried over from the last cell plus zeros): flush at these indices
    __device__ __forceinline__ void scatter_end(const DGrid& g, float* acc) const {
#pragma unroll
        for (int k = 0; k < 8; ++k) flush(g, acc, k);
    }
    // vr_transmittance_DDA.h:121-153 second march: dL/dsigma per corner
    template <bool EXACT>
    __device__ __forceinline__ void scatter(const DGrid& g, float dL_dtau, Tally& tl) {
        float acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.0f;
        float ct = 0.0f;
        int it = 0;
        const float stop = tau_stop<EXACT>();
        while (ct < stop && it < kStepCap) {
            scatter_cell<EXACT>(g, dL_dtau, acc, ct);
            tl.reds += 4;
            ++it;
        }
        tl.reds += 4;
        scatter_end(g, acc);
    }
};

template <bool EXACT>
__device__ __forceinline__ float transmittance_dda(const DMedium& M, float3 x, float3 w, Tally& tl) {
    DDA q;
    if (!q.init(M, x, w)) return 1.0f;
    return expf(-q.tau<EXACT>(M.sigma, tl));
}
template <bool EXACT>
__device__ __forceinline__ void transmittance_dda_bw(const DMedium& M, float3 x, float3 w, float dL_dT, Tally& tl) {
    if (dL_dT == 0.0f || !M.sigma.grad) return;
    DDA q;
    if (!q.init(M, x, w)) return;
    float tau = q.tau<EXACT>(M.sigma, tl);
    float T = expf(-tau);
    q.reset(M);
    q.scatter<EXACT>(M.sigma, -dL_dT * T, tl);
}

// GridRatiotrackingTransmittance / GridDeltatrackingTransmittance
// (include/vr_transmittance_GRT.h:1-83, _GDT.h:1-84): the DDA walk of the
// grid's cells (the corner values stay in registers, 4 new loads per cell);
// per cell the eight corners bound the trilinear field, the minorant part is
// integrated in closed form (exp(-min * dt)) and the residual sigma - min is
// tracked against max - min: ratio tracking multiplies T by 1 - Pc, delta
// tracking ends the ray (T = 0) at a collision.  Forward only: the
// reference's maps define no backward.
// One cell of it: the minorant part in closed form, the residual tracked to
// the cell's end.  False when the ray ends in the cell (DELTA: a collision,
// T = 0; or the step cap, error 4).
template <bool DELTA>
__device__ __forceinline__ bool grid_tracking_cell(const DMedium& M, DDA& q, Rng& rng, float& T, float& ct, int& it,
                                                   Tally& tl, uint32_t* status) {
    const float nt = gmin(q.d, gmin(q.alpha.x, gmin(q.alpha.y, q.alpha.z)));
    float mx = q.s[0], mn = q.s[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        mx = fmaxf(mx, q.s[k]);
        mn = fminf(mn, q.s[k]);
    }
    ++tl.steps;
    ++tl.lookups;
    T *= expf(-mn * (nt - ct));
    const float rm = gmax(0.000001f, mx - mn);
    float cell_t = ct;
    while (true) {
        if (++it > kStepCap) {
            raise_status(status, 4);
            return false;
        }
        const float dt = -logf(1.0f - rng.uniform()) / rm;
        if (cell_t + dt > nt) break;
        cell_t += dt;
        const float Pc = (q.interp(q.ialpha(cell_t)) - mn) / rm;
        ++tl.steps;
        if (DELTA) {
            if (rng.uniform() < Pc) {
                T = 0.0f;
                return false;
            }
        } else {
            T *= (1.0f - Pc);
        }
    }
    ct = nt;
    const int axis = q.advance_cell();
    q.shift_load(M.sigma, axis);
    return true;
}
template <bool DELTA>
__device__ __forceinline__ float transmittance_grid_tracking(const DMedium& M, Rng& rng, float3 x, float3 w,
                                                             Tally& tl, uint32_t* status) {
    DDA q;
    if (!q.init(M, x, w)) return 1.0f;
    q.load_all(M.sigma);
    float T = 1.0f, ct = 0.0f;
    const float stop = q.d - 0.0001f;
    int it = 0;
    while (ct < stop) {
        if (++it > kStepCap) {
            raise_status(status, 4);
            return T;
        }
        if (!grid_tracking_cell<DELTA>(M, q, rng, T, ct, it, tl, status)) return T;
    }
    return T;
}

// vr_transmittance_RT.h:1-49.  The "grid crossing" branch restarts at a
// majorant-brick face without a collision; it cannot trigger with the
// constant majorant (distance 1e6).
// One iteration of its loop (a brick crossing or a tracking collision): true
// when the estimate is complete (in T).
__device__ __forceinline__ bool rt_step(const DMedium& M, Rng& rng, Flight& ff, float3& x, float3 w, float& d,
                                        float& T, Tally& tl) {
    float md;
    float maj = gmax(0.0000001f, ff.bk.query(M, x, w, md));
    if (ff.tau < 0.0f) ++tl.steps;
    float t = ff.sample(rng) / maj;
    if (md < d && t > md) {
        x = x + w * md;
        d -= md;
        ff.cross(maj, md);
        ff.bk.advance(M);
        return false;
    }
    ff.used();
    float dt = gmin(t, gmin(d, md));
    ff.bk.move(dt);
    x = x + w * dt;
    d -= dt;
    if (d <= 0.0000001f) return true;
    T *= (1.0f - sigma(M, x, tl) / maj);
    if (T < 0.01f) {
        if (rng.uniform() < 1.0f - T) {
            T = 0.0f;
            return true;
        }
        T = 1.0f;
    }
    return false;
}
__device__ __forceinline__ float transmittance_rt(const DMedium& M, Rng& rng, float3 x, float3 w, Tally& tl,
                                                  uint32_t* status) {
    float T = 1.0f;
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return T;
    x = x + w * tMin;
    float d = tMax - tMin;
    Flight ff;
    for (int it = 0; it < kStepCap; ++it)
        if (rt_step(M, rng, ff, x, w, d, T, tl)) return T;
    raise_status(status, 4);
    return T;
}

// vr_transmittance_RT.h:51-141
__device__ __forceinline__ void transmittance_rt_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float dL_dT,
                                                    Tally& tl, uint32_t* status) {
    if (dL_dT == 0.0f) return;
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return;
    const float EPS = 0.0000001f;
    float T = 1.0f;
    x = x + w * tMin;
    float d = tMax - tMin;
    const float3 ini_x = x;
    const float ini_d = d;
    const Rng::Pos before = rng.pos();
    int it = 0;
    Flight ff;
    for (; it < kStepCap; ++it) {
        float md;
        float maj = gmax(EPS, ff.bk.query(M, x, w, md) + 0.1f);
        float t = ff.sample(rng) / maj;
        if (md < d && t > md) { x = x + w * md; d -= md; ff.cross(maj, md); ff.bk.advance(M); continue; }
        ff.used();
        float dt = gmin(t, gmin(d, md));
        ff.bk.move(dt);
        x = x + w * dt;
        d -= dt;
        if (d <= EPS) break;
        T *= (1.0f - sigma(M, x, tl) / maj);
        if (T < 0.1f) {
            if (rng.uniform() < 1.0f - T) return;
            T = 1.0f;
        }
    }
    if (it == kStepCap) { raise_status(status, 4); return; }
    const float out_T = T;
    T = 1.0f;
    rng.seek(before);
    x = ini_x;
    d = ini_d;
    ff = Flight();
    for (it = 0; it < kStepCap; ++it) {
        float md;
        float maj = gmax(EPS, ff.bk.query(M, x, w, md) + 0.1f);
        float t = ff.sample(rng) / maj;
        if (md < d && t > md) { x = x + w * md; d -= md; ff.cross(maj, md); ff.bk.advance(M); continue; }
        ff.used();
        float dt = gmin(t, gmin(d, md));
        ff.bk.move(dt);
        x = x + w * dt;
        d -= dt;
        if (d <= EPS) break;
        float r = (1.0f - sigma(M, x, tl) / maj);
        T *= r;
        sigma_bw(M, x, -out_T * dL_dT / maj / r, tl);
        if (T < 0.1f) {
            rng.advance();
            T = 1.0f;
        }
    }
}

// vr_transmittance_DT.h:1-28
// One iteration of its loop: 0 the ray goes on, 1 it left the segment (T = 1),
// 2 a real collision (T = 0).
__device__ __forceinline__ int dt_step(const DMedium& M, Rng& rng, Flight& ff, float3& x, float3 w, float& d,
                                       Tally& tl) {
    float md;
    float maj = gmax(0.0000001f, ff.bk.query(M, x, w, md));
    if (ff.tau < 0.0f) ++tl.steps;
    float dt = ff.sample(rng) / maj;
    float t = gmin(md, dt);
    x = x + w * t;
    d -= t;
    // the end test precedes the brick-crossing restart (the reference's
    // order, which the constant majorant never distinguishes)
    if (d <= 0.0000001f) return 1;
    if (dt > md) {
        ff.cross(maj, md);
        ff.bk.advance(M);
        return 0;
    }
    ff.used();
    ff.bk.move(t);
    if (rng.uniform() < sigma(M, x, tl) / maj) return 2;
    return 0;
}
__device__ __forceinline__ float transmittance_dt(const DMedium& M, Rng& rng, float3 x, float3 w, Tally& tl,
                                                  uint32_t* status) {
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return 1.0f;
    x = x + w * tMin;
    float d = tMax - tMin;
    Flight ff;
    for (int it = 0; it < kStepCap; ++it) {
        const int r = dt_step(M, rng, ff, x, w, d, tl);
        if (r) return r == 1 ? 1.0f : 0.0f;
    }
    raise_status(status, 4);
    return 1.0f;
}

// vr_transmittance_DT.h:30-90
__device__ __forceinline__ void transmittance_dt_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float dL_dT,
                                                    Tally& tl, uint32_t* status) {
    if (dL_dT == 0.0f) return;
    float tMin, tMax;
    if (!boundary(M, x, w, tMin, tMax)) return;
    x = x + w * tMin;
    float d = tMax - tMin;
    const float3 ini_x = x;
    const float ini_d = d;
    const Rng::Pos before = rng.pos();
    int it = 0;
    Flight ff;
    for (; it < kStepCap; ++it) {
        float md;
        float maj = gmax(0.0000001f, ff.bk.query(M, x, w, md) + 0.1f);
        float dt = ff.sample(rng) / maj;
        float t = gmin(md, dt);
        x = x + w * t;
        d -= t;
        if (d <= 0.0000001f) break;
        if (dt > md) { ff.cross(maj, md); ff.bk.advance(M); continue; }
        ff.used();
        ff.bk.move(t);
        if (rng.uniform() < sigma(M, x, tl) / maj) return;
    }
    if (it == kStepCap) { raise_status(status, 4); return; }
    x = ini_x;
    d = ini_d;
    rng.seek(before);
    ff = Flight();
    for (it = 0; it < kStepCap; ++it) {
        float md;
        float maj = gmax(0.0000001f, ff.bk.query(M, x, w, md) + 0.1f);
        float dt = ff.sample(rng) / maj;
        float t = gmin(md, dt);
        x = x + w * t;
        d -= t;
        if (d <= 0.0000001f) break;
        if (dt > md) { ff.cross(maj, md); ff.bk.advance(M); continue; }
        ff.used();
        ff.bk.move(t);
        rng.advance();
        float Pc = sigma(M, x, tl) / maj;
        sigma_bw(M, x, -dL_dT / maj / (1.0f - Pc), tl);
    }
}

// include/vr_transmittance.h dispatch over the medium's transmittance map; each
// call draws from a fork of the caller's stream
__device__ __forceinline__ float transmittance(const DMedium& M, Rng& rng, float3 x, float3 w, Tally& tl,
                                               uint32_t* status) {
    Rng sr = rng.fork();
    switch (M.tr_mode) {
        case 0: return transmittance_rt(M, sr, x, w, tl, status);
        case 1: return transmittance_dt(M, sr, x, w, tl, status);
        case 2: return transmittance_dda<false>(M, x, w, tl);
        case 3: return transmittance_dda<true>(M, x, w, tl);
        case 4: return transmittance_grid_tracking<false>(M, sr, x, w, tl, status);
        default: return transmittance_grid_tracking<true>(M, sr, x, w, tl, status);
    }
}
__device__ __forceinline__ void transmittance_bw(const DMedium& M, Rng& rng, float3 x, float3 w, float dL_dT,
                                                 Tally& tl, uint32_t* status) {
    Rng sr = rng.fork();
    switch (M.tr_mode) {
        case 0: transmittance_rt_bw(M, sr, x, w, dL_dT, tl, status); break;
        case 1: transmittance_dt_bw(M, sr, x, w, dL_dT, tl, status); break;
        case 2: transmittance_dda_bw<false>(M, x, w, dL_dT, tl); break;
        case 3: transmittance_dda_bw<true>(M, x, w, dL_dT, tl); break;
        default: break;  // GRT / GDT: no backward (the reference's maps define none)
    }
}

}  // namespace vrt
